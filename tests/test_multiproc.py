"""The multi-GPU bench path, exercised on CPU with two gloo ranks.

bench.py shards windows across ranks with no collective on the data path;
torch.distributed only provides the barrier and the max / sum over ranks of
the measured times and counters. This runs that logic with world size 2 on
the gloo backend (no GPU) and checks the reductions, the per-rank shards and
the whole-job rate.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    from poa_b200 import synth
    D = bench.Dist(world)
    try:
        D.barrier()
        t = 1.0 + rank                      # rank 1 is the slow one
        t_max = D.max(t)
        failed = D.sum(rank)                # counters add up
        ws = synth.polishing_windows(seed=bench.shard_seed(rank), n_windows=3)
        first = ws.window_reads(0)[0]
        out[rank] = (t_max, failed, ws.n_windows, first[:32])
    finally:
        D.close()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    (t0, f0, n0, r0), (t1, f1, n1, r1) = out[0], out[1]
    assert t0 == t1 == 2.0          # both ranks see the slowest rank's time
    assert f0 == f1 == 1            # 0 + 1
    assert n0 == n1 == 3            # weak scaling: the same work per rank
    assert r0 != r1                 # distinct shards
    import bench
    assert bench.whole_job_rate(world, n0, 5, t0) == pytest.approx(2 * 3 * 5 / 2.0)
