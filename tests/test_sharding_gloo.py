"""Batches of graphs split across ranks by estimated work (grappolo_b200.sharding):
each graph in exactly one shard, loads within the LPT bound, and the per-graph
results gathered back in the original order.  The multi-rank path is checked
with two gloo ranks on the CPU; each rank stands in for one GPU with a per-graph
result computed on the host."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from grappolo_b200 import graphs, sharding  # noqa: E402


def _work():
    specs = graphs.batch_specs(4096, seed=3)
    return specs[:, 0] * specs[:, 3]  # expected CSR entries: vertices x mean degree


def test_shards_cover_every_graph_once_and_balance():
    work = _work()
    for world in (1, 2, 3, 4, 8):
        shards = sharding.shard_by_work(work, world)
        allidx = np.concatenate(shards)
        assert len(allidx) == len(work) and len(np.unique(allidx)) == len(work)
        loads = sharding.shard_loads(work, shards)
        # LPT is within 4/3 of the optimum, which is at least the mean load
        assert loads.max() <= (4 / 3) * max(loads.mean(), work.max()) + 1e-9
        # on this batch (many graphs, none dominant) the split is near even
        assert loads.max() / loads.mean() < 1.01


def test_shard_is_deterministic():
    work = _work()
    a = sharding.shard_by_work(work, 4)
    b = sharding.shard_by_work(work, 4)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_gather_single_process():
    idx = np.array([2, 0, 1])
    vals = np.array([[20.0], [0.0], [10.0]])
    out = sharding.gather_results(idx, vals, 3)
    assert np.array_equal(out[:, 0], [0.0, 10.0, 20.0])


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
    from grappolo_b200 import sharding as sh
    work = _work()
    mine = sh.shard_by_work(work, world)[rank]
    # a per-graph "result" each rank computes for its own graphs only
    vals = np.stack([mine * 2.0, work[mine]], axis=1)
    full = sh.gather_results(mine, vals, len(work), dist)
    out[rank] = (full[:, 0].tolist(), float(full[:, 1].sum()), len(mine))
    dist.destroy_process_group()


def test_two_ranks_gather_in_graph_order():
    ctx = mp.get_context('spawn')
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    work = _work()
    for r in range(2):
        ids, total, n = out[r]
        assert ids == (np.arange(len(work)) * 2.0).tolist()
        assert abs(total - work.sum()) < 1e-6 * work.sum()
    assert out[0][2] + out[1][2] == len(work)
