"""Multi-rank host logic of bench.py on CPU (gloo, world size 2).

The hot path shards by independent solves: each rank solves its own batch
(disjoint density seeds, ``bench.shard_seed0``) with no exchange in the timed
region; afterwards the per-solve results (seed, V-cycles, final error, E_H)
are all-gathered (``bench.gather_results``) and the timings reduced by max.
Here each gloo rank runs that per-rank logic with the oracle's solver on
small grids, and rank 0's gathered table must equal a single-process run over
both shards, row for row.  No GPU is involved; on GPUs the same calls run
over NCCL.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N, B = 16, 2


def shard_table(rank):
    """One rank's solves: seeds from its shard, the oracle's float64 solver."""
    sys.path.insert(0, ROOT)
    import bench
    from gpawdft_b200.workloads import gaussian_density
    from oracle import layer
    from oracle.geometry import GridDescriptor
    rows = []
    for i in range(B):
        seed = bench.shard_seed0(rank) + i
        rho, L = gaussian_density(N, 0.3, 4, seed)
        gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
        ps = layer.PoissonSolver(nn=3, relax='J', eps=1e-18)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        phi = gd.zeros()
        n = ps.solve(phi, rho)
        rows.append([seed, n, ps.errors[-1],
                     0.5 * gd.dv * float(np.dot(phi.ravel(), rho.ravel()))])
    return np.array(rows)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        table = shard_table(rank)
        gathered = bench.gather_results(table, dist, 'cpu')
        t = bench.reduce_max(float(rank + 1) * 0.5, dist, 'cpu')
        q.put((rank, gathered, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_gather():
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
    res = sorted((q.get(timeout=300) for _ in range(2)), key=lambda r: r[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, g0, t0), (_, g1, t1) = res
    assert t0 == t1 == 1.0                    # max over ranks everywhere
    single = np.concatenate([shard_table(0), shard_table(1)])
    assert g0.shape == (2 * B, 4)
    assert np.array_equal(g0, single)         # rank order, row for row
    assert np.array_equal(g1, single)         # all-gather: every rank has it
    seeds = g0[:, 0]
    assert len(np.unique(seeds)) == 2 * B     # disjoint shards
    import bench
    summ = bench.results_summary(g0, None)
    assert summ['solves'] == 2 * B and summ['seeds_distinct']
    assert summ['vcycles_min'] >= 1
