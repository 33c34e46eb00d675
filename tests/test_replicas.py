"""The multi-GPU path of bench.py is replicas only: every rank runs its own
filter (its own seed), the step time is the max over ranks and the value the
particle-steps of all ranks over that time.  Checked here with two gloo ranks
on the CPU (no GPU, no collective in the data path)."""

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    import bench
    ms = 100.0 + 50.0 * rank            # rank 1 is the slower replica
    m = bench.max_over_ranks(ms, dist, 'cpu')
    seed = 1000 + rank                   # the seed bench.py gives each rank's filter
    out.put((rank, m, bench.replica_throughput(2000, world, m), seed))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_take_max_over_ranks_with_gloo():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [150.0, 150.0]
    assert res[0][2] == pytest.approx(2000 * 2 / 0.150)
    assert res[0][3] != res[1][3]
