"""Multi-rank sharding logic of bench.py on CPU (gloo, world size 2).

The hot path shards by independent solves; ranks exchange nothing but the
max of their timings.  Two gloo ranks check that their density seeds are
disjoint, their densities differ, and the max-over-ranks reduction returns
the same value everywhere.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        seed0 = bench.shard_seed0(rank)
        from gpawdft_b200.workloads import gaussian_density
        rho, _ = gaussian_density(16, 0.3, 4, seed0)
        t = bench.reduce_max(float(rank + 1) * 0.5, dist, 'cpu')
        q.put((rank, seed0, float(np.abs(rho).sum()), t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding():
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, a0, t0), (r1, s1, a1, t1) = res
    assert s0 != s1 and abs(s1 - s0) >= 1000   # disjoint seed ranges
    assert a0 != a1                            # different densities
    assert t0 == t1 == 1.0                     # max over ranks everywhere
