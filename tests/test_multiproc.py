"""The multi-GPU path, exercised on CPU with two gloo ranks.

bench.py (and poa_batch_consensus_multi in the library) split ONE window set
over the ranks by cost (poa_batch_partition), run each share with no
collective on the data path, and gather the per-window results in input
order; torch.distributed gives the barrier, the max / sum over ranks of the
measured times and counters, and the gather. Here two gloo ranks (no GPU)
run that logic on a real window list, each computing its share's consensus
with the CPU restatement in oracle/ standing in for its device, and the
gathered result must equal a single process's over the whole list.
"""
import os
import socket
import subprocess
import tempfile

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle", "build", "poa_oracle")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _consensus(ws, windows):
    from poa_b200 import synth
    out = []
    with tempfile.TemporaryDirectory() as d:
        for w in windows:
            fa = os.path.join(d, "w.fa")
            synth.write_fasta(fa, ws.window_reads(int(w)))
            out.append(subprocess.run([ORACLE, fa], capture_output=True, check=True).stdout)
    return out


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
        ws = synth.polishing_windows(seed=43, n_windows=12)
        mine = bench.rank_windows(ws, world, rank)
        cons = _consensus(ws, mine)
        gathered = bench.gather_in_order(D, mine, cons, ws.n_windows)
        out[rank] = (t_max, failed, [int(w) for w in mine], gathered)
    finally:
        D.close()


def test_two_gloo_ranks_share_one_window_set(oracle_bin):
    world, port = 2, _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    (t0, f0, m0, g0), (t1, f1, m1, g1) = out[0], out[1]
    assert t0 == t1 == 2.0          # both ranks see the slowest rank's time
    assert f0 == f1 == 1            # 0 + 1
    assert sorted(m0 + m1) == list(range(12)) and not set(m0) & set(m1)  # every window once
    assert m0 and m1                # both ranks have work
    from poa_b200 import synth
    ws = synth.polishing_windows(seed=43, n_windows=12)
    want = _consensus(ws, range(12))
    assert g0 == g1 == want         # gathered in input order, equal to one process's results
    import bench
    assert bench.whole_job_rate(12, 5, t0) == pytest.approx(12 * 5 / 2.0)
