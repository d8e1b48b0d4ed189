"""Python mirror of the reference's hot-path interface over the C ABI.

Names and argument meaning follow the reference crate (raw-lab/sabertooth
v0.4.0): GapCosts (src/align.rs:198-223), QueryProfile.from_rows / build /
sw_score / sw_score_with (src/simd.rs:128-292), Kernel (src/simd.rs:40-49,
with GPU variants), diag_range / kadane_score / Lane / DiagProfile /
score_batch (src/ungapped.rs:38-386).  Every score is computed on the GPU by
libsabertooth_b200.so; there is no CPU path.  Targets of the batched forms
are ordinals of the device-resident database (Context.upload_db).
"""
import ctypes as C
import enum
import threading
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (CANDIDATE_DTYPE, HIT_DTYPE, LANE_DTYPE, PAIR_DTYPE, PREFILTER_STATS_FIELDS, SEED_HIT_DTYPE,
                   check, lib, ptr)

ALPHABET_SIZE = 21


@dataclass(frozen=True)
class GapCosts:
    """A gap of length L costs open + (L-1)*extend."""

    open: int
    extend: int

    @staticmethod
    def sequence_default():
        return GapCosts(11, 1)

    @staticmethod
    def profile_default():
        return GapCosts(44, 4)

    def cost(self, length):
        return 0 if length == 0 else self.open + (length - 1) * self.extend


@dataclass(frozen=True)
class PrefilterParams:
    """The reference's PrefilterParams (src/prefilter.rs:262-303; defaults
    sequence_default :309-331 and profile_default :333-341): the segment-evidence
    fields, the similar-k-mer fields, and span: the seed pattern's span (k for a
    contiguous seed), which widens each diagonal's window past its last hit (taken
    from the seed index when the seeds are generated on the device)."""

    min_hits: int = 1
    min_diag_score: int = 42
    diag_hits: int = 1
    max_diagonals: int = 4
    max_candidates: int = 0
    regions: bool = False
    diag_window: int = 48
    span: int = 6
    kmer_score: int = 22
    max_kmers_per_pos: int = 512
    exact_seeds: bool = True
    max_seed_occ: int = 0

    @staticmethod
    def sequence_default():
        return PrefilterParams()

    @staticmethod
    def profile_default():
        return PrefilterParams(min_diag_score=30, span=5, kmer_score=40, exact_seeds=False)

    def seed_c(self):
        return _lib.SeedParamsC(self.kmer_score, self.max_kmers_per_pos, 1 if self.exact_seeds else 0,
                                self.max_seed_occ)

    def to_c(self, gaps: GapCosts):
        return _lib.PrefilterParamsC(self.min_hits, self.diag_hits, self.max_diagonals, self.diag_window, self.span,
                                     self.min_diag_score, gaps.open, gaps.extend, self.max_candidates,
                                     1 if self.regions else 0)


class Kernel(enum.IntEnum):
    """Which kernel produced a score."""

    NONE = 0    # empty query or target: 0 without a launch
    GPU16 = 1   # packed 16-bit DPX kernel (exact below its headroom)
    GPU32 = 2   # exact 32-bit kernel (rescore, wide rows, any gap costs, band)


def diag_range(m, n, d):
    """Query positions [lo, hi) where diagonal d = target_pos - query_pos lies in both sequences."""
    lo = max(-d, 0)
    hi = min(m, n - d)
    return (0, 0) if hi <= lo else (lo, hi)


class Context:
    """A device, its stream, the device-resident target database and query profiles."""

    def __init__(self, device=0, hbm_budget_bytes=0):
        h = lib.st_init(device, hbm_budget_bytes)
        if not h:
            raise _lib.StError(-2, lib.st_last_error().decode())
        self._h = C.c_void_p(h)
        self.device = device
        self.n_seqs = 0
        self.db_lengths = np.zeros(0, dtype=np.uint32)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib.st_shutdown(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, cuda_stream_ptr):
        """Launch on a caller-owned cudaStream_t (an int address, e.g. torch.cuda.Stream.cuda_stream)."""
        check(lib.st_set_stream(self._h, C.c_void_p(cuda_stream_ptr) if cuda_stream_ptr else None))

    def synchronize(self):
        check(lib.st_synchronize(self._h))

    def mem_used(self):
        v = C.c_uint64()
        check(lib.st_mem_used(self._h, C.byref(v)))
        return v.value

    def launch_count(self):
        v = C.c_uint64()
        check(lib.st_launch_count(self._h, C.byref(v)))
        return v.value

    # -- database ---------------------------------------------------------
    def upload_db(self, residues, offsets):
        """residues: uint8 codes; offsets: n_seqs+1 uint64 (sequence s = residues[offsets[s]:offsets[s+1]])."""
        residues = np.ascontiguousarray(residues, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        n = len(offsets) - 1
        check(lib.st_db_upload(self._h, ptr(residues) if residues.size else None, ptr(offsets), n))
        self.n_seqs = n
        self.db_lengths = np.diff(offsets).astype(np.uint32)
        # the host arena stays referenced: lanes built from db_seq() slices point into it
        self._db_host = (residues, offsets)

    def db_seq(self, i):
        """Residues of database sequence i as a view of the uploaded host arena (SeedIndex::seq,
        src/index.rs:1975-1979): the target slice a Lane carries."""
        res, offs = self._db_host
        return res[int(offs[i]):int(offs[i + 1])]

    def db_info(self):
        """(sequences, residues) of the device database."""
        n, r = C.c_uint32(), C.c_uint64()
        check(lib.st_db_info(self._h, C.byref(n), C.byref(r)))
        return n.value, r.value

    def upload_db_list(self, seqs):
        offs = np.zeros(len(seqs) + 1, dtype=np.uint64)
        offs[1:] = np.cumsum([len(s) for s in seqs])
        res = np.concatenate([np.asarray(s, dtype=np.uint8) for s in seqs]) if seqs else np.zeros(0, np.uint8)
        self.upload_db(res, offs)

    # -- profiles -----------------------------------------------------------
    def create_profiles(self, rows_list):
        """Profiles from a list of int32 [m][21] row arrays; returns their ids."""
        if not rows_list:
            return np.zeros(0, dtype=np.uint32)
        arrs = [np.ascontiguousarray(r, dtype=np.int32).reshape(-1, ALPHABET_SIZE) for r in rows_list]
        offs = np.zeros(len(arrs) + 1, dtype=np.uint64)
        offs[1:] = np.cumsum([a.shape[0] for a in arrs])
        arena = np.concatenate(arrs, axis=0) if offs[-1] else np.zeros((1, ALPHABET_SIZE), np.int32)
        arena = np.ascontiguousarray(arena)
        ids = np.zeros(len(arrs), dtype=np.uint32)
        check(lib.st_profiles_create(self._h, ptr(arena), ptr(offs), len(arrs), ptr(ids)))
        return ids

    def create_profiles_arena(self, rows_arena, row_offsets):
        """Profiles from one int32 [total_rows][21] arena; profile k = rows row_offsets[k]..row_offsets[k+1]."""
        arena = np.ascontiguousarray(rows_arena, dtype=np.int32)
        offs = np.ascontiguousarray(row_offsets, dtype=np.uint64)
        ids = np.zeros(len(offs) - 1, dtype=np.uint32)
        if len(ids):
            check(lib.st_profiles_create(self._h, ptr(arena), ptr(offs), len(ids), ptr(ids)))
        return ids

    def free_profile(self, pid):
        check(lib.st_profile_free(self._h, int(pid)))

    def free_profiles(self, ids):
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        if len(ids):
            check(lib.st_profiles_free(self._h, ptr(ids), len(ids)))

    # -- (G) batched -------------------------------------------------------
    def sw_score_pairs(self, pairs, gaps: GapCosts, with_kernels=False):
        """Scores of many (profile, db target[, band]) pairs; host buffers in and out."""
        pairs = as_pairs(pairs)
        n = len(pairs)
        scores = np.zeros(n, dtype=np.int32)
        kernels = np.zeros(n, dtype=np.uint32) if with_kernels else None
        if n:
            check(lib.st_sw_score_pairs(self._h, ptr(pairs), n, gaps.open, gaps.extend, ptr(scores),
                                        ptr(kernels)))
        return (scores, kernels) if with_kernels else scores

    def sw_score_end_pairs(self, pairs, gaps: GapCosts):
        """(scores, ends[n, 2]): score and end cell (query, target; -1 for a zero score) of every pair."""
        pairs = as_pairs(pairs)
        n = len(pairs)
        scores = np.zeros(n, dtype=np.int32)
        ends = np.zeros((n, 2), dtype=np.int32)
        if n:
            check(lib.st_sw_score_end_pairs(self._h, ptr(pairs), n, gaps.open, gaps.extend, ptr(scores), ptr(ends)))
        return scores, ends

    def align_span_pairs(self, pairs, gaps: GapCosts):
        """(scores, starts[n, 2], ends[n, 2]): the alignment span of every pair (align_canonical's two score
        passes); -1 for a zero score."""
        pairs = as_pairs(pairs)
        n = len(pairs)
        scores = np.zeros(n, dtype=np.int32)
        ends = np.zeros((n, 2), dtype=np.int32)
        starts = np.zeros((n, 2), dtype=np.int32)
        if n:
            check(lib.st_sw_align_span_pairs(self._h, ptr(pairs), n, gaps.open, gaps.extend, ptr(scores), ptr(ends),
                                             ptr(starts)))
        return scores, starts, ends

    def sw_score_pairs_async(self, pairs, gaps: GapCosts, scores=None, kernels=None, with_kernels=False):
        """Starts scoring `pairs` and returns a Batch at once; Batch.wait() returns the scores
        (and kernel tags). `scores` / `kernels` may be given (for instance pinned arrays) and
        must not be read before wait()."""
        pairs = as_pairs(pairs)
        n = len(pairs)
        if scores is None:
            scores = np.zeros(n, dtype=np.int32)
        if kernels is None and with_kernels:
            kernels = np.zeros(n, dtype=np.uint32)
        h = C.c_void_p()
        check(lib.st_sw_score_pairs_async(self._h, ptr(pairs), n, gaps.open, gaps.extend, ptr(scores),
                                          ptr(kernels), C.byref(h)))
        return Batch(h, scores, kernels)

    def plan(self, pairs, gaps: GapCosts, d_scores, d_kernels=None):
        return Plan(self, pairs, gaps, d_scores, d_kernels)

    # -- (U) ---------------------------------------------------------------
    def ungapped_hits(self, hits, with_pairs=True):
        """Per-hit best ungapped segment score, and per (query, target) run: (best, query, target)."""
        hits = as_hits(hits)
        n = len(hits)
        per_hit = np.zeros(n, dtype=np.int32)
        if not with_pairs:
            check(lib.st_ungapped_hits(self._h, ptr(hits), n, ptr(per_hit), None, None, None, None))
            return per_hit
        pb = np.zeros(max(n, 1), dtype=np.int32)
        pq = np.zeros(max(n, 1), dtype=np.uint32)
        pt = np.zeros(max(n, 1), dtype=np.uint32)
        npairs = C.c_uint64()
        check(lib.st_ungapped_hits(self._h, ptr(hits), n, ptr(per_hit), ptr(pb), ptr(pq), ptr(pt),
                                   C.byref(npairs)))
        k = npairs.value
        return per_hit, (pb[:k].copy(), pq[:k].copy(), pt[:k].copy())

    def ungapped_hits_device(self, d_hits_ptr, n, d_per_hit_ptr, d_pair_best=None, d_pair_query=None,
                             d_pair_target=None, d_n_pairs=None):
        check(lib.st_ungapped_hits_device(self._h, C.c_void_p(d_hits_ptr), n, C.c_void_p(d_per_hit_ptr),
                                          _vp(d_pair_best), _vp(d_pair_query), _vp(d_pair_target),
                                          _vp(d_n_pairs)))

    def prefilter_gate(self, hits, params: PrefilterParams = None, gaps: GapCosts = None):
        """Seed hits (query profile id, target, diagonal, query position) -> ranked
        candidates (CANDIDATE_DTYPE: per query id, score descending, target
        ascending) and the evidence counters, the reference's score_and_gate stage
        (src/prefilter.rs:1412-1660, 1074-1083) for every query of the batch."""
        hits = as_seed_hits(hits)
        params = params or PrefilterParams.sequence_default()
        gaps = gaps or GapCosts.sequence_default()
        n = len(hits)
        out = np.zeros(max(n, 1), dtype=CANDIDATE_DTYPE)
        n_out = C.c_uint64()
        st = _lib.PrefilterStatsC()
        prm = params.to_c(gaps)
        check(lib.st_prefilter_gate(self._h, ptr(hits), n, C.byref(prm), ptr(out), n, C.byref(n_out),
                                    C.byref(st)))
        return out[:n_out.value].copy(), {f: getattr(st, f) for f in PREFILTER_STATS_FIELDS}

    def seed_index_build(self, seed_mask="111001101"):
        """Indexes the device database for a seed pattern (0/1 mask; the reference's
        sequence default 111001101, profile default 11111)."""
        check(lib.st_seed_index_build(self._h, seed_mask.encode()))

    @staticmethod
    def _queries(profile_ids, residues):
        ids = np.ascontiguousarray(profile_ids, dtype=np.uint32)
        if residues is None:
            return ids, None, None
        offs = np.zeros(len(residues) + 1, dtype=np.uint64)
        offs[1:] = np.cumsum([len(r) for r in residues])
        res = np.concatenate([np.asarray(r, dtype=np.uint8) for r in residues]) if len(residues) else \
            np.zeros(1, np.uint8)
        return ids, np.ascontiguousarray(res), offs

    def seed_hits(self, profile_ids, residues=None, params: PrefilterParams = None):
        """Seed hits (SEED_HIT_DTYPE, unordered) of the queries and the seed counters;
        residues: per query its residue codes (sequence queries) or None (profiles)."""
        params = params or PrefilterParams.sequence_default()
        ids, res, offs = self._queries(profile_ids, residues)
        sp = params.seed_c()
        st = _lib.SeedStatsC()
        n = C.c_uint64()
        args = (self._h, ptr(ids), len(ids), ptr(res) if res is not None else None,
                ptr(offs) if offs is not None else None, C.byref(sp))
        check(lib.st_seed_hits(*args, None, 0, C.byref(n), C.byref(st)))
        out = np.zeros(max(n.value, 1), dtype=SEED_HIT_DTYPE)
        check(lib.st_seed_hits(*args, ptr(out), n.value, C.byref(n), C.byref(st)))
        return out[:n.value].copy(), {f: getattr(st, f) for f in _lib.SEED_STATS_FIELDS}

    def prefilter_queries(self, profile_ids, residues=None, params: PrefilterParams = None, gaps: GapCosts = None):
        """The whole prefilter of the queries on the device (seed hits -> evidence ->
        chains -> gate -> ranking): candidates (CANDIDATE_DTYPE), evidence counters,
        seed counters."""
        params = params or PrefilterParams.sequence_default()
        gaps = gaps or GapCosts.sequence_default()
        ids, res, offs = self._queries(profile_ids, residues)
        sp = params.seed_c()
        gp = params.to_c(gaps)
        st = _lib.PrefilterStatsC()
        sst = _lib.SeedStatsC()
        n = C.c_uint64()
        args = (self._h, ptr(ids), len(ids), ptr(res) if res is not None else None,
                ptr(offs) if offs is not None else None, C.byref(sp), C.byref(gp))
        cap = max(1 << 16, 1024 * len(ids))  # a batch with more candidates runs again with the exact room
        while True:
            out = np.empty(cap, dtype=CANDIDATE_DTYPE)
            check(lib.st_prefilter_queries(*args, ptr(out), cap, C.byref(n), C.byref(st), C.byref(sst)))
            if n.value <= cap:
                break
            cap = int(n.value)
        return (out[:n.value].copy(), {f: getattr(st, f) for f in PREFILTER_STATS_FIELDS},
                {f: getattr(sst, f) for f in _lib.SEED_STATS_FIELDS})

    def prefilter_gate_device(self, d_hits_ptr, n, d_out_ptr, params: PrefilterParams = None,
                              gaps: GapCosts = None):
        """Device-buffer form: returns (candidate count, counters); d_out has room for n candidates."""
        params = params or PrefilterParams.sequence_default()
        gaps = gaps or GapCosts.sequence_default()
        n_out = C.c_uint64()
        st = _lib.PrefilterStatsC()
        prm = params.to_c(gaps)
        check(lib.st_prefilter_gate_device(self._h, C.c_void_p(d_hits_ptr), n, C.byref(prm), C.c_void_p(d_out_ptr),
                                           C.byref(n_out), C.byref(st)))
        return n_out.value, {f: getattr(st, f) for f in PREFILTER_STATS_FIELDS}

    def calibrate_profiles(self, profile_ids, lengths, samples=2000, seed=0x5EED, gaps: GapCosts = None,
                           p_back=None, with_scores=False):
        """calibrate_profile (src/evalue.rs:714-748) for each profile id: a list of
        (lambda, k, mu) per profile, None where the reference returns None.  All
        profiles are scored against the same `samples` background targets (the
        reference's per-search seed 0x5EED and database length sample); the
        scoring runs on the GPU, the maximum-likelihood fits on the host."""
        ids = np.ascontiguousarray(profile_ids, dtype=np.uint32)
        lengths = np.ascontiguousarray(lengths, dtype=np.uint32)
        gaps = gaps or GapCosts.profile_default()
        if p_back is None:
            from .matrix import blosum62
            p_back = blosum62().p_back[:20]
        pb = np.ascontiguousarray(p_back, dtype=np.float64)
        out = (_lib.CalibrationC * max(len(ids), 1))()
        sc = np.zeros((len(ids), samples), dtype=np.int32) if with_scores else None
        check(lib.st_calibrate_profiles(self._h, ptr(ids), len(ids), ptr(lengths) if len(lengths) else None,
                                        len(lengths), samples, seed, ptr(pb), gaps.open, gaps.extend,
                                        ptr(sc) if sc is not None and sc.size else None, out))
        res = [(o.lambda_, o.k, o.mu) if o.ok else None for o in out[:len(ids)]]
        return (res, sc) if with_scores else res

    # -- tuning / measurement ---------------------------------------------------
    def autotune(self, pairs, gaps: GapCosts, max_pairs=200_000):
        """Measures every tile class's rate on a sample of `pairs`; returns the number of classes measured."""
        pairs = as_pairs(pairs)
        nb = C.c_uint32()
        check(lib.st_autotune(self._h, ptr(pairs), len(pairs), gaps.open, gaps.extend, max_pairs, C.byref(nb)))
        return nb.value

    def tuning_table(self):
        t = np.zeros((10, 8), dtype=np.int32)
        check(lib.st_tune_get(self._h, ptr(t)))
        return t

    def set_tuning_table(self, table):
        t = np.ascontiguousarray(table, dtype=np.int32).reshape(10, 8)
        check(lib.st_tune_set(self._h, ptr(t)))

    def tuning_rates(self):
        r = np.zeros(lib.st_tune_num_classes(), dtype=np.float32)
        check(lib.st_tune_get_rates(self._h, ptr(r), len(r)))
        return r

    def set_tuning_rates(self, rates):
        r = np.ascontiguousarray(rates, dtype=np.float32)
        check(lib.st_tune_set_rates(self._h, ptr(r), len(r)))

    def probe_dpx(self):
        v = C.c_double()
        check(lib.st_probe_dpx(self._h, C.byref(v)))
        return v.value


def _vp(x):
    return C.c_void_p(x) if x else None


def tile_classes():
    """(lanes per alignment G, query rows per lane R, target columns per step C) of every tile class."""
    out = []
    for c in range(lib.st_tune_num_classes()):
        g, r, k = C.c_int(), C.c_int(), C.c_int()
        check(lib.st_tune_class_shape(c, C.byref(g), C.byref(r), C.byref(k)))
        out.append((g.value, r.value, k.value))
    return out


def as_pairs(pairs):
    if isinstance(pairs, np.ndarray) and pairs.dtype == PAIR_DTYPE:
        return np.ascontiguousarray(pairs)
    arr = np.zeros(len(pairs), dtype=PAIR_DTYPE)
    for i, p in enumerate(pairs):
        prof, tgt = p[0], p[1]
        c, r = (p[2], p[3]) if len(p) > 2 else (0, -1)
        arr[i] = (prof, tgt, c, r)
    return arr


def as_hits(hits):
    if isinstance(hits, np.ndarray) and hits.dtype == HIT_DTYPE:
        return np.ascontiguousarray(hits)
    arr = np.zeros(len(hits), dtype=HIT_DTYPE)
    for i, h in enumerate(hits):
        arr[i] = tuple(h)
    return arr


def as_seed_hits(hits):
    if isinstance(hits, np.ndarray) and hits.dtype == SEED_HIT_DTYPE:
        return np.ascontiguousarray(hits)
    arr = np.zeros(len(hits), dtype=SEED_HIT_DTYPE)
    for i, h in enumerate(hits):
        arr[i] = tuple(h)
    return arr


class Batch:
    """A batch started by Context.sw_score_pairs_async; wait() exactly once."""

    def __init__(self, handle, scores, kernels):
        self._h = handle
        self.scores = scores
        self.kernels = kernels

    def wait(self):
        if self._h is None:
            raise RuntimeError("batch already waited for")
        h, self._h = self._h, None
        check(lib.st_batch_wait(h))
        return (self.scores, self.kernels) if self.kernels is not None else self.scores

    def __del__(self):
        if getattr(self, "_h", None) is not None:
            try:
                lib.st_batch_wait(self._h)
            except Exception:
                pass


class Server:
    """Continuous batching of scoring requests (st_server_*): submit() returns a request id at
    once, wait(id) returns (scores, latency_ms). One worker thread per server batches requests
    in arrival order and keeps two batches in flight."""

    def __init__(self, ctx: Context, gaps: GapCosts, max_batch_pairs=0, hbm_budget_bytes=0):
        self._ctx = ctx
        self._h = lib.st_server_create(ctx.handle, gaps.open, gaps.extend, int(max_batch_pairs),
                                       int(hbm_budget_bytes))
        if not self._h:
            check(-1)
        self._n = {}

    def submit(self, rows, targets, band_center=None, band_radius=None):
        rows = np.ascontiguousarray(rows, dtype=np.int32).reshape(-1, 21)
        targets = np.ascontiguousarray(targets, dtype=np.uint32)
        bc = None if band_center is None else np.ascontiguousarray(band_center, dtype=np.int32)
        br = None if band_radius is None else np.ascontiguousarray(band_radius, dtype=np.int32)
        rid = C.c_uint64()
        check(lib.st_server_submit(self._h, ptr(rows), rows.shape[0], ptr(targets), ptr(bc), ptr(br),
                                   len(targets), C.byref(rid)))
        self._n[rid.value] = len(targets)
        return rid.value

    def submit_many(self, rows_arena, row_offsets, targets, target_offsets, band_center=None, band_radius=None):
        """Requests arriving together: request k = rows_arena[row_offsets[k]:row_offsets[k+1]] against
        targets[target_offsets[k]:target_offsets[k+1]]. Returns the request ids."""
        rows = np.ascontiguousarray(rows_arena, dtype=np.int32).reshape(-1, 21)
        ro = np.ascontiguousarray(row_offsets, dtype=np.uint64)
        t = np.ascontiguousarray(targets, dtype=np.uint32)
        to = np.ascontiguousarray(target_offsets, dtype=np.uint64)
        bc = None if band_center is None else np.ascontiguousarray(band_center, dtype=np.int32)
        br = None if band_radius is None else np.ascontiguousarray(band_radius, dtype=np.int32)
        k = len(ro) - 1
        ids = np.zeros(k, dtype=np.uint64)
        check(lib.st_server_submit_many(self._h, k, ptr(rows), ptr(ro), ptr(t), ptr(to), ptr(bc), ptr(br), ptr(ids)))
        for j in range(k):
            self._n[int(ids[j])] = int(to[j + 1] - to[j])
        return ids

    def wait(self, rid):
        n = self._n.pop(int(rid))
        out = np.zeros(n, dtype=np.int32)
        lat = C.c_double()
        check(lib.st_server_wait(self._h, int(rid), ptr(out), n, C.byref(lat)))
        return out, lat.value

    def stats(self):
        b, p = C.c_uint64(), C.c_uint64()
        check(lib.st_server_stats(self._h, C.byref(b), C.byref(p)))
        return {"batches": b.value, "pairs": p.value}

    def close(self):
        if self._h:
            lib.st_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SearchServer:
    """Whole searches as a service (st_search_server_*): submit(rows, residues) returns a request
    id at once; wait(id) returns (candidates, SW scores, latency_ms). One worker thread runs the
    requests that have arrived as one batch: seeds -> evidence -> gate -> SW on the device."""

    def __init__(self, ctx: Context, params: "PrefilterParams" = None, gaps: GapCosts = None, sequence_queries=True,
                 max_batch_queries=0):
        params = params or PrefilterParams.sequence_default()
        gaps = gaps or GapCosts.sequence_default()
        self._ctx = ctx
        self._sp = params.seed_c()
        self._gp = params.to_c(gaps)
        self._h = lib.st_search_server_create(ctx.handle, C.byref(self._sp), C.byref(self._gp),
                                              1 if sequence_queries else 0, int(max_batch_queries))
        if not self._h:
            check(-1)

    def submit(self, rows, residues=None):
        rows = np.ascontiguousarray(rows, dtype=np.int32).reshape(-1, 21)
        res = None if residues is None else np.ascontiguousarray(residues, dtype=np.uint8)
        rid = C.c_uint64()
        check(lib.st_search_server_submit(self._h, ptr(rows), rows.shape[0], ptr(res), C.byref(rid)))
        return rid.value

    def wait(self, rid):
        n = C.c_uint64()
        lat = C.c_double()
        cap = 4096
        while True:
            out = np.zeros(cap, dtype=CANDIDATE_DTYPE)
            sc = np.zeros(cap, dtype=np.int32)
            check(lib.st_search_server_wait(self._h, int(rid), ptr(out), ptr(sc), cap, C.byref(n), C.byref(lat)))
            if n.value <= cap:
                return out[:n.value].copy(), sc[:n.value].copy(), lat.value
            cap = int(n.value)

    def stats(self):
        b, q = C.c_uint64(), C.c_uint64()
        check(lib.st_search_server_stats(self._h, C.byref(b), C.byref(q)))
        return {"batches": b.value, "queries": q.value}

    def close(self):
        if self._h:
            lib.st_search_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """A captured batch over device buffers (d_scores / d_kernels: device pointers as ints)."""

    def __init__(self, ctx: Context, pairs, gaps: GapCosts, d_scores, d_kernels=None):
        pairs = as_pairs(pairs)
        self.ctx = ctx
        self.n = len(pairs)
        h = C.c_void_p()
        check(lib.st_plan_create(ctx.handle, ptr(pairs), self.n, gaps.open, gaps.extend, C.c_void_p(d_scores),
                                 _vp(d_kernels), C.byref(h)))
        self._h = h

    def run(self):
        check(lib.st_plan_run(self._h))

    def stats(self):
        cells, resc, ncls = C.c_uint64(), C.c_uint64(), C.c_uint32()
        check(lib.st_plan_stats(self._h, C.byref(cells), C.byref(resc), C.byref(ncls)))
        return {"cells": cells.value, "rescored_pairs": resc.value, "launch_classes": ncls.value}

    def profile(self):
        """Each launch alone: [(tile class (G, R, C), or "sw32" for the 32-bit kernel, or "band16" for the packed
        kernel of banded pairs, cells, ms)]."""
        cap = 32
        cls = np.zeros(cap, dtype=np.int32)
        cells = np.zeros(cap, dtype=np.uint64)
        ms = np.zeros(cap, dtype=np.float32)
        n = C.c_uint32()
        check(lib.st_plan_profile(self._h, cap, ptr(cls), ptr(cells), ptr(ms), C.byref(n)))
        shapes = tile_classes()
        names = {-1: "sw32", -2: "band16"}
        return [(shapes[cls[i]] if cls[i] >= 0 else names[int(cls[i])], int(cells[i]), float(ms[i]))
                for i in range(n.value)]

    def close(self):
        if self._h:
            lib.st_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# -- process-wide default context (like the reference's process-wide kernel choice) --
_default = None
_default_lock = threading.Lock()


def default_context() -> Context:
    global _default
    with _default_lock:
        if _default is None:
            _default = Context(0)
        return _default


class QueryProfile:
    """A query (sequence or PSSM) prepared for repeated scoring (src/simd.rs:128-139)."""

    def __init__(self, rows, ctx: Context = None):
        self.ctx = ctx or default_context()
        self._rows = np.ascontiguousarray(rows, dtype=np.int32).reshape(-1, ALPHABET_SIZE)
        self.m = self._rows.shape[0]
        self.id = int(self.ctx.create_profiles([self._rows])[0])

    @staticmethod
    def from_rows(rows, ctx: Context = None):
        return QueryProfile(rows, ctx)

    @staticmethod
    def build(scorer_rows, ctx: Context = None):
        return QueryProfile(scorer_rows, ctx)

    def query_len(self):
        return self.m

    def rows(self):
        return self._rows

    def sw_score(self, target, gaps: GapCosts) -> int:
        return self.sw_score_with(target, gaps)[0]

    def sw_score_end(self, target, gaps: GapCosts):
        """QueryProfile::sw_score_end_with: (score, query end, target end), or None for a zero score."""
        t = np.ascontiguousarray(target, dtype=np.uint8)
        s, qe, te = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib.st_sw_score_end(self.ctx.handle, self.id, ptr(t) if t.size else None, t.size, gaps.open,
                                  gaps.extend, C.byref(s), C.byref(qe), C.byref(te)))
        return None if s.value <= 0 else (s.value, qe.value, te.value)

    def sw_score_with(self, target, gaps: GapCosts, scratch=None):
        """(score, Kernel) of one host target: the plain per-call drop-in."""
        t = np.ascontiguousarray(target, dtype=np.uint8)
        s, k = C.c_int32(), C.c_uint32()
        check(lib.st_sw_score(self.ctx.handle, self.id, ptr(t) if t.size else None, t.size, gaps.open,
                              gaps.extend, C.byref(s), C.byref(k)))
        return s.value, Kernel(k.value)

    def free(self):
        self.ctx.free_profile(self.id)


@dataclass
class Lane:
    """One diagonal job (src/ungapped.rs:265-270): the target, the diagonal and the query window [lo, hi).

    As in the reference, `target` is a slice of a database sequence: a uint8 view of the host arena that was
    uploaded (Context.db_seq(i), or any sub-slice of it).  A database ordinal (int) is accepted too."""

    target: object
    diag: int
    lo: int
    hi: int


class DiagProfile:
    """Ungapped scoring profile of a query (src/ungapped.rs:188-255); any score range works on the GPU."""

    def __init__(self, qp: QueryProfile):
        self.qp = qp

    @staticmethod
    def build(rows, ctx: Context = None):
        if len(rows) == 0:
            return None  # the reference refuses empty profiles too (src/ungapped.rs:225)
        return DiagProfile(QueryProfile(rows, ctx))

    def query_len(self):
        return self.qp.m


def score_batch(prof: DiagProfile, lanes, out=None):
    """out[i] = best ungapped segment score of lanes[i] (src/ungapped.rs:285-386), any number of lanes.
    Lanes whose targets are arena slices go through st_ungapped_score_slices (the reference's Lane as it
    is); lanes with database ordinals through st_ungapped_score."""
    n = len(lanes)
    res = np.zeros(n, dtype=np.int32)
    if n and isinstance(lanes[0].target, np.ndarray):
        arr = (_lib.st_lane_slice * n)()
        for i, l in enumerate(lanes):
            t = l.target
            if not isinstance(t, np.ndarray) or t.dtype != np.uint8 or (t.size and not t.flags.c_contiguous):
                raise TypeError("every lane's target must be a contiguous uint8 slice of the uploaded arena")
            arr[i] = _lib.st_lane_slice(t.ctypes.data if t.size else 0, t.size, l.diag, l.lo, l.hi)
        check(lib.st_ungapped_score_slices(prof.qp.ctx.handle, prof.qp.id, arr, n, ptr(res)))
    elif n:
        arr = np.zeros(n, dtype=LANE_DTYPE)
        for i, l in enumerate(lanes):
            arr[i] = (l.target, l.lo, l.hi, l.diag)
        check(lib.st_ungapped_score(prof.qp.ctx.handle, prof.qp.id, ptr(arr), n, ptr(res)))
    if out is not None:
        out[:n] = res
    return res


def kadane_score(prof: DiagProfile, target, d, lo, hi) -> int:
    """Best ungapped segment of one diagonal window (src/ungapped.rs:53-62), on the GPU."""
    return int(score_batch(prof, [Lane(target, d, lo, hi)])[0])
