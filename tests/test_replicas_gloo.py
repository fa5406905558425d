"""Multi-GPU form of the benchmark: independent replicas, no data-path
collective; whole-job time is the max over ranks and the edges are summed.
Checked with two gloo ranks on the CPU."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    t, e = bench.aggregate(1.0 + rank, 100.0 * (rank + 1), dist, 'cpu')
    out[rank] = (t, e)
    dist.destroy_process_group()


def test_replica_aggregation_two_ranks():
    ctx = mp.get_context('spawn')
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == (2.0, 300.0) and out[1] == (2.0, 300.0)


def test_single_process_passthrough():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate(3.0, 7.0) == (3.0, 7.0)
