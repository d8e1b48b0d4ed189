"""The N > 1 path of bench.py on CPU: two ranks over gloo (127.0.0.1). Each rank scores its own
instance of the workload (seed + rank: weak scaling, no collective on the data path); the job's
step time is the slowest rank's and its work the sum of the ranks'."""
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
    w = bench.make_workload(A, r)
    ms, cells = bench.combine_ranks(10.0 + r, w.cells(), "cpu")
    out[rank] = (ms, cells, w.cells(), int(sum(len(r) for r in w.rows)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_weak_scaling_max_over_ranks():
    port = _free_port()
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    (ms0, c0, own0, sig0), (ms1, c1, own1, sig1) = out[0], out[1]
    assert ms0 == ms1 == 11.0  # the slowest rank's step time
    assert c0 == c1 == float(own0 + own1)  # the whole job's work
    assert sig0 != sig1  # each rank scores its own instance (seed + rank)
