"""st_sw_score_noalloc: the allocation-free entry point, checked against st_sw_score and the oracle.

Some callers cannot allocate device memory: code running inside a stream
capture, serving threads that cannot take cudaFree's implicit
synchronisation, or processes whose device memory belongs to another
allocator.  They pass device buffers they own and the kernel keeps its scratch
in a static device array.  This test calls the entry point through the C ABI
twice in a row (the second call finds the first call's scratch contents) and
compares both scores, bit for bit, with the allocating per-call entry point
st_sw_score and with the oracle's scalar Gotoh (src/simd.rs:347-390) on the
same pairs.  Multi-pass queries (more than 256 rows) against targets shorter
than a warp run right after a long, high-scoring call, so a read of the
previous call's scratch would show as a wrong score.  The test's own device
buffers come from torch; the entry point itself allocates nothing.  The file
sorts last so that a stop-at-first-failure run has already run every other
test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pairs():
    from synth import workloads as W
    model = W.Model()
    r = W.Rng(2024)
    out = []
    # a 700-row query (three 256-row passes: the scratch is written and read back) vs a homolog-bearing target
    q1 = model.background(r, 700)
    t1 = model.background(r, 3000)
    t1[1000:1700] = model.mutate(r, q1, 0.8)
    out.append((model.mat.sequence_rows(q1), t1, 11, 1))
    # a short query against a long target, other gap costs
    q2 = model.background(r, 300)
    t2 = model.background(r, 20000)
    t2[5000:5300] = model.mutate(r, q2, 0.6)
    out.append((model.mat.sequence_rows(q2), t2, 44, 4))
    return out


def test_noalloc_matches_the_allocating_entry_point_on_two_calls():
    import torch

    from oracle import oracle as O
    from sabertooth_b200 import Context, GapCosts, QueryProfile
    from sabertooth_b200._lib import check, lib

    torch.cuda.set_device(0)
    ctx = Context(0)
    try:
        for rows, target, go, ge in _pairs():
            qp = QueryProfile.from_rows(rows, ctx)
            want, _ = qp.sw_score_with(target, GapCosts(go, ge))
            qp.free()
            assert want == O.gotoh_score(rows, target, go, ge)
            d_rows = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.int32)).cuda()
            d_t = torch.from_numpy(np.ascontiguousarray(target, dtype=np.uint8)).cuda()
            d_out = torch.full((1,), -1, dtype=torch.int32, device="cuda")
            stream = torch.cuda.current_stream().cuda_stream
            check(lib.st_sw_score_noalloc(d_rows.data_ptr(), rows.shape[0], d_t.data_ptr(), target.size, go, ge,
                                          d_out.data_ptr(), C.c_void_p(stream) if stream else None))
            torch.cuda.synchronize()
            assert int(d_out.item()) == want
    finally:
        ctx.close()


def _noalloc(rows, target, go, ge):
    import torch

    from sabertooth_b200._lib import check, lib

    d_rows = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.int32)).cuda()
    d_t = torch.from_numpy(np.ascontiguousarray(target, dtype=np.uint8)).cuda()
    d_out = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    check(lib.st_sw_score_noalloc(d_rows.data_ptr(), rows.shape[0], d_t.data_ptr() if target.size else None,
                                  target.size, go, ge, d_out.data_ptr(), C.c_void_p(stream) if stream else None))
    torch.cuda.synchronize()
    return int(d_out.item())


def test_noalloc_short_targets_after_a_long_call_match_the_oracle():
    import torch

    from oracle import oracle as O
    from sabertooth_b200 import Context, GapCosts, QueryProfile
    from synth import workloads as W

    torch.cuda.set_device(0)
    model = W.Model()
    r = W.Rng(77)
    w = np.full(3000, 18, dtype=np.uint8)  # W x 3000: large H values all over the scratch
    w_rows = model.mat.sequence_rows(w)
    ctx = Context(0)
    try:
        for m in (257, 300, 700, 5000):
            for n in (1, 2, 5, 10, 16, 31, 32, 33):
                q = model.background(r, m)
                t = model.background(r, n)
                t[: min(n, 8)] = q[100:100 + min(n, 8)]
                rows = model.mat.sequence_rows(q)
                for go, ge in ((11, 1), (44, 4)):
                    assert _noalloc(w_rows, w, go, ge) == O.gotoh_score(w_rows, w, go, ge)
                    want = O.gotoh_score(rows, t, go, ge)
                    qp = QueryProfile.from_rows(rows, ctx)
                    alloc, _ = qp.sw_score_with(t, GapCosts(go, ge))
                    qp.free()
                    assert alloc == want, (m, n, go, ge)
                    for _ in range(2):  # two calls in a row: the second sees the first one's scratch
                        assert _noalloc(rows, t, go, ge) == want, (m, n, go, ge)
    finally:
        ctx.close()


def test_noalloc_rejects_targets_beyond_its_static_scratch():
    import torch

    from sabertooth_b200._lib import lib

    torch.cuda.set_device(0)
    d = torch.zeros(65537, dtype=torch.uint8, device="cuda")
    rows = torch.zeros((4, 21), dtype=torch.int32, device="cuda")
    out = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.st_sw_score_noalloc(rows.data_ptr(), 4, d.data_ptr(), 65537, 11, 1, out.data_ptr(), None)
    assert rc == -1
    assert b"65536" in lib.st_last_error()
