"""Seeded synthetic workloads with the shapes of the five benchmark configurations.

The reference benchmarks on ASTRAL SCOPe40 plus Markov filler, which is not
available here; these generators stand in with the same sizes, length
distributions and residue composition:

* residues i.i.d. from the BLOSUM62 background (the reference's
  BackgroundSampler, src/evalue.rs:85-114);
* lengths median * exp(sigma * N(0,1)), clipped;
* planted homologs: each site keeps the source residue with probability p,
  otherwise draws from P(b|a) = prob[a][b] / p_back[a] (src/matrix.rs:137-151),
  with geometric indels;
* PSSM queries from 50-member family MSAs (40-90% identity) through the
  reference's PSSM construction (synth.profile).

Random numbers come from SplitMix64 (src/evalue.rs:54-75) evaluated in counter
form: output i of a stream seeded s is mix(s + (i+1)*gamma), so whole arrays
are drawn at once and every workload is reproducible from its seed.
"""
from dataclasses import dataclass, field

import numpy as np

from sabertooth_b200.matrix import PROFILE_AA_SIZE, blosum62

GAMMA = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def _mix(z):
    z = (z ^ (z >> np.uint64(30))) * M1
    z = (z ^ (z >> np.uint64(27))) * M2
    return z ^ (z >> np.uint64(31))


class Rng:
    """Counter-form SplitMix64: each draw of n values consumes n outputs of the stream."""

    def __init__(self, seed):
        self.state = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
        self.count = 0

    def u64(self, n):
        with np.errstate(over="ignore"):
            idx = np.arange(self.count + 1, self.count + 1 + n, dtype=np.uint64)
            out = _mix(self.state + idx * GAMMA)
        self.count += n
        return out

    def uniform(self, n):
        return (self.u64(n) >> np.uint64(11)).astype(np.float64) / float(1 << 53)

    def below(self, n, k):
        return (self.u64(n) % np.uint64(k)).astype(np.int64)

    def normal(self, n):
        u1 = np.maximum(self.uniform(n), 1e-300)
        u2 = self.uniform(n)
        return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)

    def child(self, k):
        with np.errstate(over="ignore"):
            s = _mix(self.state ^ (np.uint64(k) * np.uint64(0xA24BAED4963EE407)) ^ np.uint64(0x9FB21C651E98DF25))
        return Rng(int(s))


class Model:
    """Residue composition and substitution model from the BLOSUM62 reconstruction."""

    def __init__(self, mat=None):
        self.mat = mat or blosum62()
        pb = self.mat.p_back[:PROFILE_AA_SIZE]
        self.cum = np.cumsum(pb / pb.sum())
        self.cum[-1] = 1.0
        cond = self.mat.prob[:PROFILE_AA_SIZE, :PROFILE_AA_SIZE] / self.mat.p_back[:PROFILE_AA_SIZE, None]
        cond = cond / cond.sum(axis=1, keepdims=True)
        self.cond_cum = np.cumsum(cond, axis=1)
        self.cond_cum[:, -1] = 1.0

    def background(self, rng: Rng, n):
        return np.searchsorted(self.cum, rng.uniform(n), side="right").astype(np.uint8)

    def substitute(self, rng: Rng, src):
        """One BLOSUM62-conditional draw per site."""
        src = np.asarray(src, dtype=np.uint8)
        u = rng.uniform(src.size)
        out = np.empty(src.size, dtype=np.uint8)
        for a in range(PROFILE_AA_SIZE):
            sel = src == a
            if sel.any():
                out[sel] = np.searchsorted(self.cond_cum[a], u[sel], side="right")
        other = src >= PROFILE_AA_SIZE
        out[other] = src[other]
        return out

    def mutate(self, rng: Rng, src, keep, indel_rate=0.0, indel_mean=2.0):
        """Keep each site with probability `keep`, else substitute; geometric indels at indel_rate/site."""
        src = np.asarray(src, dtype=np.uint8)
        n = src.size
        sub = self.substitute(rng, src)
        k = rng.uniform(n) < keep
        out = np.where(k, src, sub).astype(np.uint8)
        if indel_rate <= 0 or n == 0:
            return out
        ev = rng.uniform(n)
        ins = ev < indel_rate / 2
        dele = (ev >= indel_rate / 2) & (ev < indel_rate)
        p = 1.0 / indel_mean
        glen = 1 + np.floor(np.log(np.maximum(rng.uniform(n), 1e-300)) / np.log(1.0 - p)).astype(np.int64)
        keep_mask = np.ones(n, dtype=bool)
        for i in np.nonzero(dele)[0]:
            keep_mask[i:i + glen[i]] = False
        pieces, last = [], 0
        ins_idx = np.nonzero(ins & keep_mask)[0]
        extra = self.background(rng, int(glen[ins_idx].sum()) if ins_idx.size else 0)
        eo = 0
        for i in ins_idx:
            pieces.append(out[last:i][keep_mask[last:i]])
            pieces.append(extra[eo:eo + glen[i]])
            eo += glen[i]
            last = i
        pieces.append(out[last:][keep_mask[last:]])
        return np.concatenate(pieces).astype(np.uint8)


def lognormal_lengths(rng: Rng, n, median, sigma, lo, hi):
    x = median * np.exp(sigma * rng.normal(n))
    return np.clip(np.rint(x), lo, hi).astype(np.int64)


def loguniform_lengths(rng: Rng, n, lo, hi):
    x = np.exp(np.log(lo) + (np.log(hi) - np.log(lo)) * rng.uniform(n))
    return np.clip(np.rint(x), lo, hi).astype(np.int64)


def pack(seqs):
    offs = np.zeros(len(seqs) + 1, dtype=np.uint64)
    if seqs:
        offs[1:] = np.cumsum([len(s) for s in seqs])
    res = np.concatenate(seqs).astype(np.uint8) if seqs and offs[-1] else np.zeros(0, np.uint8)
    return res, offs


@dataclass
class SwWorkload:
    """Query rows, a target database and (query, target[, band]) pairs with one gap setting."""

    name: str
    rows: list                     # int32 [m][21] per query
    db_residues: np.ndarray        # uint8 arena
    db_offsets: np.ndarray         # uint64 [n+1]
    pair_q: np.ndarray             # uint32
    pair_t: np.ndarray             # uint32
    gap_open: int
    gap_extend: int
    band_center: np.ndarray = None  # int32, with band_radius
    band_radius: np.ndarray = None  # int32, -1 = full
    info: dict = field(default_factory=dict)

    @property
    def n_pairs(self):
        return len(self.pair_q)

    def targets(self):
        o = self.db_offsets
        return [self.db_residues[int(o[i]):int(o[i + 1])] for i in range(len(o) - 1)]

    def cells(self):
        """The reference's gapped_cells: sum of m*n over full pairs (src/search.rs:538); band cells for banded pairs."""
        m = np.array([len(r) for r in self.rows], dtype=np.int64)[self.pair_q]
        n = np.diff(self.db_offsets.astype(np.int64))[self.pair_t]
        if self.band_radius is None:
            return int((m * n).sum())
        full = self.band_radius < 0
        tot = int((m[full] * n[full]).sum())
        for k in np.nonzero(~full)[0]:
            tot += band_cells(int(m[k]), int(n[k]), int(self.band_center[k]), int(self.band_radius[k]))
        return tot

    def cells_of(self, i):
        """Cells of pair i (m*n, or band cells for a banded pair)."""
        m = len(self.rows[int(self.pair_q[i])])
        n = int(self.db_offsets[int(self.pair_t[i]) + 1] - self.db_offsets[int(self.pair_t[i])])
        if self.band_radius is None or self.band_radius[i] < 0:
            return m * n
        return band_cells(m, n, int(self.band_center[i]), int(self.band_radius[i]))


def band_cells(m, n, center, radius):
    i = np.arange(1, m + 1, dtype=np.int64)
    lo = np.maximum(1, i + center - radius)
    hi = np.minimum(n, i + center + radius)
    return int(np.maximum(hi - lo + 1, 0).sum())


def seq_rows(model: Model, q):
    return model.mat.sequence_rows(q)


def pssm_rows(pssm):
    r = np.zeros((pssm.shape[0], 21), dtype=np.int32)
    r[:, :PROFILE_AA_SIZE] = pssm
    return r


# ---- config 1: plain exhaustive SW (BLOSUM62, 11/1) -------------------------
def config1(seed=0, n_queries=200, n_targets=20000, homolog_frac=0.10, identity=0.40, model=None):
    model = model or Model()
    rng = Rng(seed)
    ql = lognormal_lengths(rng, n_queries, 250, 0.5, 30, 1000)
    queries = [model.background(rng.child(i), int(l)) for i, l in enumerate(ql)]
    tl = lognormal_lengths(rng, n_targets, 250, 0.5, 30, 1000)
    hom = rng.uniform(n_targets) < homolog_frac
    src_q = rng.below(n_targets, n_queries)
    targets = []
    for t in range(n_targets):
        r = rng.child(1_000_000 + t)
        if hom[t]:
            targets.append(model.mutate(r, queries[src_q[t]], identity, indel_rate=0.02))
        else:
            targets.append(model.background(r, int(tl[t])))
    res, offs = pack(targets)
    pq = np.repeat(np.arange(n_queries, dtype=np.uint32), n_targets)
    pt = np.tile(np.arange(n_targets, dtype=np.uint32), n_queries)
    return SwWorkload("config1-exhaustive-blosum62", [seq_rows(model, q) for q in queries], res, offs, pq, pt, 11, 1,
                      info={"queries": n_queries, "targets": n_targets, "seed": seed})


# ---- config 3: PSSM queries, top-300 targets each (44/4) --------------------
def family_msa(model: Model, rng: Rng, query, members=50, id_lo=0.40, id_hi=0.90, gap_rate=0.01):
    L = query.size
    ident = id_lo + (id_hi - id_lo) * rng.uniform(members - 1)
    src = np.broadcast_to(query, (members - 1, L)).ravel()
    sub = model.substitute(rng, src).reshape(members - 1, L)
    keep = rng.uniform((members - 1) * L).reshape(members - 1, L) < ident[:, None]
    rows = np.where(keep, query[None, :], sub).astype(np.uint8)
    # deletions relative to the query appear as gap runs (1-6 columns) in the members
    starts = np.nonzero(rng.uniform((members - 1) * L) < gap_rate)[0]
    lens = 1 + rng.below(max(starts.size, 1), 6)[:starts.size]
    flat = rows.ravel()
    for s, g in zip(starts, lens):
        e = min(s + g, (s // L + 1) * L)
        flat[s:e] = 0xFF
    msa = np.empty((members, L), dtype=np.uint8)
    msa[0] = query
    msa[1:] = flat.reshape(members - 1, L)
    return msa


def config3(seed=0, n_queries=4000, db_residues=2_600_000, per_query=300, planted_per_query=2, members=50,
            model=None, threads=0):
    from .profile import pssm_batch
    model = model or Model()
    rng = Rng(seed)
    ql = loguniform_lengths(rng, n_queries, 50, 2000)
    queries = [model.background(rng.child(i), int(l)) for i, l in enumerate(ql)]
    msas = [family_msa(model, rng.child(10_000_000 + i), q, members) for i, q in enumerate(queries)]
    pssms = pssm_batch(msas, model.mat, threads=threads)
    rows = [pssm_rows(p) for p in pssms]
    # database: planted homolog fragments of each family, then background sequences up to the residue budget
    seqs, owner = [], []
    for i, q in enumerate(queries):
        r = rng.child(20_000_000 + i)
        for h in range(planted_per_query):
            flen = int(lognormal_lengths(r, 1, 182, 0.5, 30, 1000)[0])
            flen = min(flen, q.size)
            start = int(r.below(1, q.size - flen + 1)[0])
            ident = 0.40 + 0.50 * float(r.uniform(1)[0])
            seqs.append(model.mutate(r, q[start:start + flen], ident, indel_rate=0.02))
            owner.append(i)
    used = sum(len(s) for s in seqs)
    bg_rng = rng.child(30_000_000)
    k = 0
    while used < db_residues:
        l = int(lognormal_lengths(bg_rng, 1, 160, 0.55, 30, 1000)[0])
        seqs.append(model.background(bg_rng, l))
        owner.append(-1)
        used += l
        k += 1
    n_db = len(seqs)
    res, offs = pack(seqs)
    owner = np.array(owner, dtype=np.int64)
    pq_list, pt_list = [], []
    pick_rng = rng.child(40_000_000)
    for i in range(n_queries):
        own = np.nonzero(owner == i)[0] if planted_per_query else np.zeros(0, np.int64)
        want = max(0, min(per_query - own.size, n_db - own.size))  # a small database caps the targets per query
        cand = pick_rng.below(want * 2 + 16, n_db)
        cand = np.unique(cand[~np.isin(cand, own)])[:want]
        while cand.size < want:
            extra = pick_rng.below(want, n_db)
            cand = np.unique(np.concatenate([cand, extra[~np.isin(extra, own)]]))[:want]
        tg = np.concatenate([own, cand]).astype(np.uint32)
        pq_list.append(np.full(tg.size, i, dtype=np.uint32))
        pt_list.append(tg)
    return SwWorkload("config3-pssm-top300", rows, res, offs, np.concatenate(pq_list), np.concatenate(pt_list), 44, 4,
                      info={"queries": n_queries, "db_seqs": n_db, "db_residues": int(offs[-1]), "seed": seed,
                            "per_query": per_query})


# ---- config 4: long targets, near-identical pairs, band 64 -----------------
def config4(seed=0, n_pairs=50000, near_identical=0.05, radius=64, model=None, threads=0, kind="blosum62"):
    """One half of the long/overflow mix: kind 'blosum62' (11/1) or 'pssm' (44/4)."""
    from .profile import pssm_batch
    model = model or Model()
    rng = Rng(seed + (0 if kind == "blosum62" else 7919))
    n_pairs = int(n_pairs)
    ql = lognormal_lengths(rng, n_pairs, 250, 0.5, 30, 2000)
    long_t = rng.uniform(n_pairs) < 0.10
    tl = np.where(long_t, loguniform_lengths(rng, n_pairs, 10_001, 35_000), loguniform_lengths(rng, n_pairs, 1000, 10_000))
    planted = rng.uniform(n_pairs) < near_identical
    queries, targets, centers = [], [], []
    for i in range(n_pairs):
        r = rng.child(i)
        q = model.background(r, int(ql[i]))
        t = model.background(r, int(tl[i]))
        c = 0
        if planted[i]:
            pos = int(r.below(1, max(1, t.size - q.size))[0])
            t[pos:pos + q.size] = model.mutate(r, q, 0.97)[: t.size - pos]
            c = pos
        queries.append(q)
        targets.append(t)
        centers.append(c)
    if kind == "pssm":
        msas = [family_msa(model, rng.child(5_000_000 + i), q, 20) for i, q in enumerate(queries)]
        rows = [pssm_rows(p) for p in pssm_batch(msas, model.mat, threads=threads)]
        go, ge = 44, 4
    else:
        rows = [seq_rows(model, q) for q in queries]
        go, ge = 11, 1
    res, offs = pack(targets)
    ratio = tl / np.maximum(ql, 1)
    band = ratio > 4
    bc = np.where(band, np.array(centers), 0).astype(np.int32)
    br = np.where(band, radius, -1).astype(np.int32)
    idx = np.arange(n_pairs, dtype=np.uint32)
    return SwWorkload(f"config4-long-overflow-{kind}", rows, res, offs, idx, idx.copy(), go, ge, bc, br,
                      info={"pairs": n_pairs, "banded": int(band.sum()), "planted": int(planted.sum()), "seed": seed})


# ---- config 2: ungapped diagonal scoring of seed hits -----------------------
@dataclass
class HitWorkload:
    name: str
    rows: list
    db_residues: np.ndarray
    db_offsets: np.ndarray
    hits: np.ndarray  # HIT_DTYPE, sorted by (query, target)
    info: dict = field(default_factory=dict)

    def algorithmic_bytes(self):
        """Residue bytes of every scored window + 12 B per hit record + 4 B per output."""
        m = np.array([len(r) for r in self.rows], dtype=np.int64)[self.hits["query"]]
        n = np.diff(self.db_offsets.astype(np.int64))[self.hits["target"]]
        d = self.hits["diag"].astype(np.int64)
        lo = np.maximum(-d, 0)
        hi = np.minimum(m, n - d)
        return int(np.maximum(hi - lo, 0).sum()) + 16 * len(self.hits)


def config2(seed=0, n_queries=1000, n_targets=374_000, n_hits=20_000_000, homolog_frac=0.10, homolog_hit_frac=0.30,
            model=None):
    from sabertooth_b200.dtypes import HIT_DTYPE
    model = model or Model()
    rng = Rng(seed)
    ql = lognormal_lengths(rng, n_queries, 250, 0.5, 30, 1000)
    queries = [model.background(rng.child(i), int(l)) for i, l in enumerate(ql)]
    tl = lognormal_lengths(rng, n_targets, 160, 0.55, 30, 1000)
    hom = rng.uniform(n_targets) < homolog_frac
    src_q = rng.below(n_targets, n_queries)
    # targets: background, homologs keep a copy of the source query at a recorded diagonal
    total = int(tl.sum())
    arena = model.background(rng.child(99), total)
    offs = np.zeros(n_targets + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(tl)
    hom_diag = np.zeros(n_targets, dtype=np.int64)
    hr = rng.child(98)
    for t in np.nonzero(hom)[0]:
        q = queries[src_q[t]]
        n = int(tl[t])
        a = int(offs[t])
        L = min(q.size, n)
        qs = int(hr.below(1, q.size - L + 1)[0])
        ts = int(hr.below(1, n - L + 1)[0])
        arena[a + ts:a + ts + L] = model.mutate(hr, q[qs:qs + L], 0.40)
        hom_diag[t] = ts - qs
    n_hom_hits = int(n_hits * homolog_hit_frac)
    n_rand = n_hits - n_hom_hits
    hom_t = np.nonzero(hom)[0]
    # homolog hits: the planted diagonal +- a small offset
    ht = hom_t[rng.below(n_hom_hits, hom_t.size)]
    hq = src_q[ht]
    hd = hom_diag[ht] + rng.below(n_hom_hits, 7) - 3
    # random hits: uniform valid diagonals of random pairs
    rq = rng.below(n_rand, n_queries)
    rt = rng.below(n_rand, n_targets)
    m_r = ql[rq]
    n_r = tl[rt]
    rd = -(m_r - 1) + (rng.u64(n_rand) % (m_r + n_r - 1).astype(np.uint64)).astype(np.int64)
    q_all = np.concatenate([hq, rq]).astype(np.uint32)
    t_all = np.concatenate([ht, rt]).astype(np.uint32)
    d_all = np.concatenate([hd, rd]).astype(np.int32)
    order = np.lexsort((d_all, t_all, q_all))
    hits = np.zeros(n_hits, dtype=HIT_DTYPE)
    hits["query"] = q_all[order]
    hits["target"] = t_all[order]
    hits["diag"] = d_all[order]
    return HitWorkload("config2-ungapped-hits", [seq_rows(model, q) for q in queries], arena, offs, hits,
                       info={"queries": n_queries, "targets": n_targets, "hits": n_hits, "db_residues": total,
                             "seed": seed})


# ---- seed hits for the evidence / chain / gate stage -------------------------
@dataclass
class SeedHitWorkload:
    name: str
    rows: list
    db_residues: np.ndarray
    db_offsets: np.ndarray
    hits: np.ndarray  # SEED_HIT_DTYPE, in generation order (not sorted)
    info: dict = field(default_factory=dict)


def seed_hits(seed=0, n_queries=1000, n_targets=374_000, n_hits=20_000_000, homolog_frac=0.10,
              homolog_hit_frac=0.30, keep=0.55, max_gap=12, model=None):
    """Seed hits with query positions on the config-2 database shape.  Each
    homolog target holds a copy of a random query segment in two pieces on
    diagonals that differ by an insertion or deletion of 1..max_gap residues
    (substitutions keep `keep` of the sites); homolog hits lie on either
    piece's diagonal at a position inside that piece, the rest are uniform over
    random (query, target, valid diagonal, position on it)."""
    from sabertooth_b200.dtypes import SEED_HIT_DTYPE
    model = model or Model()
    rng = Rng(seed)
    ql = lognormal_lengths(rng, n_queries, 250, 0.5, 30, 1000)
    queries = [model.background(rng.child(i), int(l)) for i, l in enumerate(ql)]
    tl = lognormal_lengths(rng, n_targets, 160, 0.55, 30, 1000)
    hom = rng.uniform(n_targets) < homolog_frac
    src_q = rng.below(n_targets, n_queries)
    total = int(tl.sum())
    arena = model.background(rng.child(99), total)
    offs = np.zeros(n_targets + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(tl)
    hom_t = np.nonzero(hom)[0]
    # piece k of target t: query positions [pq0, pq1) on diagonal pd
    pq0 = np.zeros((n_targets, 2), dtype=np.int64)
    pq1 = np.zeros((n_targets, 2), dtype=np.int64)
    pd = np.zeros((n_targets, 2), dtype=np.int64)
    hr = rng.child(98)
    for t in hom_t:
        q = queries[src_q[t]]
        n = int(tl[t])
        a = int(offs[t])
        L = min(q.size, n) - max_gap
        if L < 20:
            continue
        qs = int(hr.below(1, q.size - L + 1)[0])
        g = int(hr.below(1, 2 * max_gap + 1)[0]) - max_gap  # > 0: insertion in the target, < 0: deletion
        g = g if g != 0 else 1
        ts = int(hr.below(1, n - L - max(g, 0) + 1)[0])
        cut = L // 2
        seg = model.mutate(hr, q[qs:qs + L], keep)
        # piece 0: q[qs, qs+cut) at ts; piece 1 continues after the indel
        arena[a + ts:a + ts + cut] = seg[:cut]
        if g > 0:
            arena[a + ts + cut:a + ts + cut + g] = model.background(hr, g)
            q1, t1 = qs + cut, ts + cut + g
        else:
            q1, t1 = qs + cut - g, ts + cut
        l1 = min(qs + L - q1, n - t1)
        arena[a + t1:a + t1 + l1] = seg[q1 - qs:q1 - qs + l1]
        pq0[t] = (qs, q1)
        pq1[t] = (qs + cut, q1 + l1)
        pd[t] = (ts - qs, t1 - q1)
    hom_t = hom_t[pq1[hom_t, 0] > pq0[hom_t, 0]]
    n_hom = int(n_hits * homolog_hit_frac) if hom_t.size else 0
    n_rand = n_hits - n_hom
    ht = hom_t[rng.below(n_hom, max(hom_t.size, 1))] if n_hom else np.zeros(0, np.int64)
    piece = rng.below(n_hom, 2)
    a0 = pq0[ht, piece]
    a1 = pq1[ht, piece]
    hqp = a0 + (rng.u64(n_hom) % np.maximum(a1 - a0, 1).astype(np.uint64)).astype(np.int64)
    hd = pd[ht, piece]
    hq = src_q[ht]
    rq = rng.below(n_rand, n_queries)
    rt = rng.below(n_rand, n_targets)
    m_r = ql[rq]
    n_r = tl[rt]
    rd = -(m_r - 1) + (rng.u64(n_rand) % (m_r + n_r - 1).astype(np.uint64)).astype(np.int64)
    lo = np.maximum(-rd, 0)
    hi = np.minimum(m_r, n_r - rd)
    rqp = lo + (rng.u64(n_rand) % np.maximum(hi - lo, 1).astype(np.uint64)).astype(np.int64)
    hits = np.zeros(n_hom + n_rand, dtype=SEED_HIT_DTYPE)
    hits["query"] = np.concatenate([hq, rq]).astype(np.uint32)
    hits["target"] = np.concatenate([ht, rt]).astype(np.uint32)
    hits["diag"] = np.concatenate([hd, rd]).astype(np.int32)
    hits["qpos"] = np.concatenate([hqp, rqp]).astype(np.uint32)
    perm = np.argsort(rng.u64(hits.size), kind="stable")
    return SeedHitWorkload("seed-hits-gate", [seq_rows(model, q) for q in queries], arena, offs, hits[perm],
                           info={"queries": n_queries, "targets": n_targets, "hits": int(hits.size),
                                 "db_residues": total, "homolog_targets": int(hom_t.size), "seed": seed})


# ---- config 5: whole searches (seeds -> gate -> SW) ---------------------------
@dataclass
class SearchWorkload:
    name: str
    queries: list       # uint8 residue codes per query
    rows: list          # int32 [m][21] BLOSUM62 rows per query
    db_residues: np.ndarray
    db_offsets: np.ndarray
    info: dict = field(default_factory=dict)


def size_adjusted_gate(gate, db_residues):
    """size_adjusted_gate (src/prefilter.rs:253-257): the gate of a 10^8-residue
    database moved by 2.5 (below) or 1.0 (above) per e-fold of database size,
    rounded half away from zero and clamped to 20..60."""
    x = np.log(max(db_residues, 1) / 1.0e8)
    slope = 2.5 if x < 0 else 1.0
    v = gate + slope * x
    r = np.floor(abs(v) + 0.5) * np.sign(v)
    return int(min(max(r, 20), 60))


def config5(seed=0, n_queries=1000, n_targets=1_000_000, homologs_per_query=5, keep=0.5, model=None):
    """Config 5's search workload: a database of n_targets sequences (lognormal
    median 250, sigma 0.35, clipped 30-1,000: about 265 M residues for 10^6
    targets) and sequence queries (lognormal median 250, sigma 0.5, clipped
    30-5,000); each query has homologs_per_query mutated copies (BLOSUM62-
    conditional substitutions keeping `keep` of the sites, indels at 2 % per site)
    planted into random targets."""
    model = model or Model()
    rng = Rng(seed)
    ql = lognormal_lengths(rng, n_queries, 250, 0.5, 30, 5000)
    queries = [model.background(rng.child(i), int(l)) for i, l in enumerate(ql)]
    tl = lognormal_lengths(rng, n_targets, 250, 0.35, 30, 1000)
    offs = np.zeros(n_targets + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(tl)
    total = int(offs[-1])
    arena = np.empty(total, dtype=np.uint8)
    chunk = 1 << 24
    for k, a in enumerate(range(0, total, chunk)):
        b = min(total, a + chunk)
        arena[a:b] = model.background(rng.child(10_000_000 + k), b - a)
    hr = rng.child(98)
    picks = hr.below(n_queries * homologs_per_query, n_targets)
    for j, t in enumerate(picks):
        q = queries[j // homologs_per_query]
        h = model.mutate(hr, q, keep, indel_rate=0.02)
        n = int(tl[t])
        L = min(h.size, n)
        s = int(hr.below(1, n - L + 1)[0])
        u = int(hr.below(1, h.size - L + 1)[0])
        arena[int(offs[t]) + s:int(offs[t]) + s + L] = h[u:u + L]
    return SearchWorkload("config5-search", queries, [seq_rows(model, q) for q in queries], arena, offs,
                          info={"queries": n_queries, "targets": n_targets, "db_residues": total,
                                "homologs_per_query": homologs_per_query, "seed": seed})
