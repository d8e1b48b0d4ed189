"""Oracle of the per-profile calibration (calibrate_profile, src/evalue.rs:714-748),
pinned on the CPU by the reference's own tests:

* gumbel_ml_recovers_known_parameters (src/evalue.rs:791-804): the ML fit on
  20,000 Gumbel draws from SplitMix64(1) recovers lambda 0.27 / mu 31;
* profile_calibration_is_per_profile (src/evalue.rs:893-914): two PSSMs, 1,500
  samples, seed 5, lengths 100 + 7i, gaps 44/4: gapped lambda below ln2/8 and
  materially different E-values;
* the background stream against a literal Python restatement of SplitMix64,
  stream_seed and BackgroundSampler (src/evalue.rs:53-114).
"""
import math

import numpy as np

import oracle.oracle as O
from sabertooth_b200 import blosum62
from synth.profile import Profile
from tests.refrng import SplitMix64

MSA_A = ">a\nMKVLLACDEFGHIKLMNPQRSTVWYACDEFGHIK\n>b\nMKILLSCDEFGHLKLMNPQRSTVWFACDEYGHIK\n"
MSA_B = ">a\nWWWWCCCCWWWWCCCCWWWWCCCCWWWWCCCCWW\n"


def test_gumbel_ml_recovers_known_parameters():
    rng = SplitMix64(1)
    lam, mu = 0.27, 31.0
    xs = [mu - math.log(-math.log(max(rng.next_f64(), 1e-300))) / lam for _ in range(20000)]
    f = O.fit_gumbel_ml(xs)
    assert abs(f[0] - lam) / lam < 0.03
    assert abs(f[1] - mu) < 0.2
    assert O.fit_gumbel_ml(xs[:9]) is None
    assert O.fit_gumbel_ml([5.0] * 50) is None


def _py_target(lengths, seed, i, p_back):
    total = sum(float(p) for p in p_back)
    cum, acc = [], 0.0
    for p in p_back:
        acc += float(p) / total
        cum.append(acc)
    cum[-1] = 1.0
    s = SplitMix64(seed ^ ((0xBEEF * 0xA24BAED4963EE407) & (2**64 - 1)) ^ ((i * 0x9FB21C651E98DF25) & (2**64 - 1)))
    rng = SplitMix64(s.next_u64())
    n = max(int(lengths[rng.below(len(lengths))]), 1)
    out = []
    for _ in range(n):
        u = rng.next_f64()
        out.append(next((k for k, c in enumerate(cum) if u < c), 19))
    return np.array(out, dtype=np.uint8)


def test_background_stream_matches_literal_restatement():
    pb = blosum62().p_back[:20]
    lengths = [0, 3, 17, 250, 31]
    for seed in (5, 0x5EED):
        for i in (0, 1, 2, 77, 1999):
            assert np.array_equal(O.calibration_target(lengths, seed, i, pb), _py_target(lengths, seed, i, pb))


def test_profile_calibration_is_per_profile():
    m = blosum62()
    pa = Profile.from_msa_str(MSA_A, m)
    pb = Profile.from_msa_str(MSA_B, m)
    lens = [100 + 7 * i for i in range(50)]
    (la, ka, _), _ = O.calibrate_profile(pa.rows(), lens, 1500, 5, m.p_back[:20], 44, 4)
    (lb, kb, _), _ = O.calibrate_profile(pb.rows(), lens, 1500, 5, m.p_back[:20], 44, 4)
    assert la < math.log(2) / 8 * 1.05
    # EValueParams::from_params(g, 1_000_000, 4000).evalue(300, query_len): K * m * N * exp(-lambda * 300)
    ea = ka * pa.query_len * 1e6 * math.exp(-la * 300)
    eb = kb * pb.query_len * 1e6 * math.exp(-lb * 300)
    assert abs(math.log(ea / eb)) > 0.5


def test_no_lengths_or_empty_profile_is_none():
    pb = blosum62().p_back[:20]
    rows = blosum62().sequence_rows(np.arange(20, dtype=np.uint8))
    assert O.calibrate_profile(rows, [], 100, 1, pb, 11, 1)[0] is None
    assert O.calibrate_profile(np.zeros((0, 21), np.int32), [50], 100, 1, pb, 11, 1)[0] is None
    assert O.calibrate_profile(rows, [50], 9, 1, pb, 11, 1)[0] is None
