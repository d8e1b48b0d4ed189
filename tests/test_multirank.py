"""The N > 1 path of bench.py on CPU: two ranks over gloo (127.0.0.1). Every rank builds the same
config-3 workload and takes the pairs whose target lies in its residue-balanced shard; the shares
partition the batch, and the job's step time is the slowest rank's (the max reduction of bench.py)."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    # loopback only: the container's hostname may not resolve
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), GLOO_SOCKET_IFNAME="lo")
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    import bench
    r, wsz, local = bench.dist_env()
    assert (r, wsz, local) == (rank, world, rank)

    class A:
        scale, seed = 0.002, 5
    w = bench.make_workload(A, 0)
    from sabertooth_b200.dtypes import PAIR_DTYPE
    from sabertooth_b200.shard import ShardMap
    pairs = np.zeros(w.n_pairs, dtype=PAIR_DTYPE)
    pairs["profile"] = w.pair_q
    pairs["target"] = w.pair_t
    idx, local = ShardMap.of(w.db_offsets, world).route(pairs, r)
    ms, cells = bench.combine_ranks(10.0 + r, len(idx), "cpu")
    out[rank] = (ms, cells, w.n_pairs, idx.tolist())
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_split_one_batch_by_target_shard():
    port = _free_port()
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    (ms0, c0, n0, idx0), (ms1, c1, n1, idx1) = out[0], out[1]
    assert ms0 == ms1 == 11.0  # the slowest rank's step time
    assert n0 == n1 and c0 == c1 == float(n0)  # the same batch on both ranks, split between them
    assert len(idx0) and len(idx1) and not set(idx0) & set(idx1)
    assert sorted(idx0 + idx1) == list(range(n0))
