"""PSSM query profiles (reference src/profile.rs): an input generator.

parse_msa restates src/profile.rs:372-449; the numeric PSSM construction runs
in synth/libsynth.so (st_pssm_from_msa, synth/pssm.cpp), which restates
Profile::from_numeric_msa in the reference's f32 operation order.  The kernels
take any int32 score rows; this module makes the PSSM rows of the synthetic
workloads and is pinned by the reference's demo/family.pssm.
"""
import numpy as np

from . import _lib
from sabertooth_b200.matrix import AA2NUM, ALPHABET_SIZE, GAP, PROFILE_AA_SIZE, blosum62

PCA_DEFAULT, PCB_DEFAULT, SCORE_BIAS_DEFAULT = 1.0, 1.5, 0.0  # src/profile.rs:56-65


def parse_msa(data: str):
    """Aligned FASTA or a3m -> (numeric rows [n][L] uint8 with 0xFF gaps, L)."""
    raw, cur, started = [], [], False
    for line in data.splitlines():
        line = line.rstrip()
        if line.startswith(">"):
            if started:
                raw.append("".join(cur))
                cur = []
            started = True
        else:
            cur.append(line.strip())
    if started:
        raw.append("".join(cur))
    if not raw:
        raise ValueError("MSA contains no sequences")
    is_a3m = any(ch.islower() for s in raw for ch in s)
    msa = []
    if is_a3m:
        for s in raw:
            row = []
            for ch in s:
                if ch.islower():
                    continue
                if ch in "-.":
                    row.append(GAP)
                elif ch.isupper():
                    row.append(int(AA2NUM[ord(ch)]))
            msa.append(row)
    else:
        width = max(len(s) for s in raw)
        first = raw[0]
        cols = [i for i in range(width) if i < len(first) and first[i] not in "-."]
        for s in raw:
            row = []
            for i in cols:
                ch = s[i] if i < len(s) else "-"
                row.append(GAP if ch in "-." else int(AA2NUM[ord(ch.upper())]))
            msa.append(row)
    L = len(msa[0])
    for k, row in enumerate(msa):
        if len(row) != L:
            raise ValueError(f"MSA row {k + 1} has {len(row)} match columns, expected {L}")
    return np.array(msa, dtype=np.uint8).reshape(len(msa), L), L


class Profile:
    """An int8 PSSM (query_len x 20) with its query residues (src/profile.rs:31-46)."""

    def __init__(self, pssm, neff, query_num):
        self.pssm = pssm
        self.neff = neff
        self.query_num = query_num
        self.query_len = pssm.shape[0]

    @staticmethod
    def from_numeric_msa(msa, mat=None, pca=PCA_DEFAULT, pcb=PCB_DEFAULT, score_bias=SCORE_BIAS_DEFAULT):
        mat = mat or blosum62()
        msa = np.ascontiguousarray(msa, dtype=np.uint8)
        n, L = msa.shape
        if n == 0 or L == 0:
            raise ValueError("cannot build a profile from an empty MSA")
        pssm = np.zeros((L, PROFILE_AA_SIZE), dtype=np.int8)
        neff = np.zeros(L, dtype=np.float32)
        r = np.ascontiguousarray(mat.r, dtype=np.float32)
        pb = np.ascontiguousarray(mat.p_back, dtype=np.float64)
        rc = _lib.lib.st_pssm_from_msa(_lib.ptr(msa), n, L, _lib.ptr(r), _lib.ptr(pb), pca, pcb, score_bias,
                                       _lib.ptr(pssm), _lib.ptr(neff))
        if rc != 0:
            raise ValueError("PSSM construction failed")
        return Profile(pssm, neff, msa[0].copy())

    @staticmethod
    def from_msa_str(data: str, mat=None, **kw):
        msa, _ = parse_msa(data)
        return Profile.from_numeric_msa(msa, mat, **kw)

    def rows(self) -> np.ndarray:
        """ScoreTable rows: pssm[i][r] for r < 20 and 0 for X (Profile::score, src/profile.rs:72-79)."""
        out = np.zeros((self.query_len, ALPHABET_SIZE), dtype=np.int32)
        out[:, :PROFILE_AA_SIZE] = self.pssm
        return out


def pssm_batch(msas, mat=None, pca=PCA_DEFAULT, pcb=PCB_DEFAULT, score_bias=SCORE_BIAS_DEFAULT, threads=0):
    """PSSMs of many numeric MSAs (list of [n_k][L_k] uint8), built in parallel on the host."""
    import os
    mat = mat or blosum62()
    n_msas = len(msas)
    rows = np.array([m.shape[0] for m in msas], dtype=np.uint32)
    lens = np.array([m.shape[1] for m in msas], dtype=np.uint32)
    sizes = rows.astype(np.uint64) * lens
    msa_off = np.zeros(n_msas, dtype=np.uint64)
    msa_off[1:] = np.cumsum(sizes)[:-1]
    arena = np.concatenate([np.ascontiguousarray(m, dtype=np.uint8).ravel() for m in msas]) if n_msas else \
        np.zeros(1, np.uint8)
    pssm_off = np.zeros(n_msas, dtype=np.uint64)
    pssm_off[1:] = np.cumsum(lens.astype(np.uint64) * PROFILE_AA_SIZE)[:-1]
    out = np.zeros(int(lens.sum()) * PROFILE_AA_SIZE + 1, dtype=np.int8)
    r = np.ascontiguousarray(mat.r, dtype=np.float32)
    pb = np.ascontiguousarray(mat.p_back, dtype=np.float64)
    nt = threads or os.cpu_count() or 1
    rc = _lib.lib.st_pssm_batch(_lib.ptr(arena), _lib.ptr(msa_off), _lib.ptr(rows), _lib.ptr(lens), n_msas,
                                _lib.ptr(r), _lib.ptr(pb), pca, pcb, score_bias, _lib.ptr(out),
                                _lib.ptr(pssm_off), nt)
    if rc != 0:
        raise ValueError("PSSM construction failed")
    return [out[int(o):int(o) + int(L) * PROFILE_AA_SIZE].reshape(int(L), PROFILE_AA_SIZE)
            for o, L in zip(pssm_off, lens)]
