"""The GPU kernels against the reference's own recorded search output.

The 88 hits of tests/data/v1_fixture_k2.v03.m8 (tests/reference_outputs.py):
the batched path and the plain per-call path score each whole pair and each
alignment span, with the rows the reference's search builds, and must print
the reference's raw score.  Rows with the composition-bias correction fit
int8, so the batched pairs run on the packed 16-bit kernel.
"""
import numpy as np
import pytest

from sabertooth_b200 import GapCosts, QueryProfile
from sabertooth_b200._lib import PAIR_DTYPE
from tests.reference_outputs import v1_fixture_cases

pytestmark = pytest.mark.gpu


def test_batched_and_per_call_scores_equal_the_recorded_raw_scores(ctx):
    cases = v1_fixture_cases()
    want = np.array([s for *_, s, _ in cases], dtype=np.int32)
    rows = [r for r, *_ in cases] + [r[q0:q1] for r, _, (q0, q1, _, _), _, _ in cases]
    targets = [t for _, t, *_ in cases] + [t[t0:t1] for _, t, (_, _, t0, t1), _, _ in cases]
    ctx.upload_db_list(targets)
    ids = ctx.create_profiles(rows)
    pairs = np.zeros(len(rows), dtype=PAIR_DTYPE)
    pairs["profile"] = ids
    pairs["target"] = np.arange(len(rows))
    pairs["band_radius"] = -1
    try:
        got, kinds = ctx.sw_score_pairs(pairs, GapCosts(11, 1), with_kernels=True)
    finally:
        ctx.free_profiles(ids)
    assert np.array_equal(got[:88], want) and np.array_equal(got[88:], want)
    assert (kinds == 1).sum() > 0
    for (r, t, _, s, _) in cases[::4]:
        qp = QueryProfile.from_rows(r, ctx)
        assert qp.sw_score(t, GapCosts(11, 1)) == s
        qp.free()
