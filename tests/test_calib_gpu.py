"""GPU parity of the per-profile calibration (st_calibrate_profiles) against the
oracle: the background scores bit for bit, the Gumbel fits (binary64, the same
summation order and libm on both sides) to a relative 1e-12, the reference's
per-profile test, the cases where the reference returns None, and the
database restored after the call.
"""
import math

import numpy as np
import pytest

import oracle.oracle as O
from sabertooth_b200 import GapCosts, blosum62
from synth import workloads as W
from synth.profile import Profile
from tests.test_calib import MSA_A, MSA_B

pytestmark = pytest.mark.gpu

REL = 1e-12


def _close(a, b):
    return abs(a - b) <= REL * max(abs(a), abs(b), 1e-300)


def test_scores_and_fits_match_oracle(ctx):
    m = blosum62()
    rng = np.random.default_rng(4)
    rows = [m.sequence_rows(rng.integers(0, 20, int(k)).astype(np.uint8)) for k in (40, 130, 333)]
    rows.append(Profile.from_msa_str(MSA_A, m).rows())
    lens = [int(x) for x in rng.integers(30, 900, 300)]
    ids = ctx.create_profiles(rows)
    try:
        for gaps in (GapCosts(44, 4), GapCosts(11, 1)):
            got, sc = ctx.calibrate_profiles(ids, lens, samples=600, seed=0x5EED, gaps=gaps, with_scores=True)
            for k, r in enumerate(rows):
                want, wsc = O.calibrate_profile(r, lens, 600, 0x5EED, m.p_back[:20], gaps.open, gaps.extend)
                assert np.array_equal(sc[k], wsc), k
                assert got[k] is not None and want is not None
                for a, b in zip(got[k], want):
                    assert _close(a, b), (k, got[k], want)
    finally:
        ctx.free_profiles(ids)


def test_reference_per_profile_calibration(ctx):
    # src/evalue.rs:893-914 on the GPU path
    m = blosum62()
    pa = Profile.from_msa_str(MSA_A, m)
    pb = Profile.from_msa_str(MSA_B, m)
    ids = ctx.create_profiles([pa.rows(), pb.rows()])
    try:
        lens = [100 + 7 * i for i in range(50)]
        (la, ka, _), (lb, kb, _) = ctx.calibrate_profiles(ids, lens, samples=1500, seed=5, gaps=GapCosts(44, 4))
        assert la < math.log(2) / 8 * 1.05
        ea = ka * pa.query_len * 1e6 * math.exp(-la * 300)
        eb = kb * pb.query_len * 1e6 * math.exp(-lb * 300)
        assert abs(math.log(ea / eb)) > 0.5
    finally:
        ctx.free_profiles(ids)


def test_none_cases_and_database_restored(ctx):
    w = W.config1(seed=6, n_queries=4, n_targets=200)
    ctx.upload_db(w.db_residues, w.db_offsets)
    ids = ctx.create_profiles(list(w.rows) + [np.zeros((0, 21), np.int32)])
    try:
        pairs = [(int(ids[q]), t) for q in range(4) for t in range(0, 200, 7)]
        before = ctx.sw_score_pairs(pairs, GapCosts(11, 1))
        assert ctx.calibrate_profiles(ids[:2], [], samples=100) == [None, None]
        res = ctx.calibrate_profiles(ids, [120, 250], samples=200, seed=3)
        assert res[-1] is None and all(r is not None for r in res[:-1])
        assert ctx.calibrate_profiles(ids[:1], [120], samples=9) == [None]
        after = ctx.sw_score_pairs(pairs, GapCosts(11, 1))
        assert np.array_equal(before, after)
        n_seqs, n_res = ctx.db_info()
        assert n_seqs == 200
    finally:
        ctx.free_profiles(ids)
