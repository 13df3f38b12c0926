"""Replica timing reduction of bench.py on two gloo ranks (CPU): every rank runs its own replica
of the workload; the job's time is the max over ranks and its scored poses the sum."""
import os
import socket

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    t, s = bench.reduce_max_sum(dist, 10.0 * (rank + 1), 100 * (rank + 1), "cpu")
    q.put((rank, t, s))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_reduction_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 20.0, 300), (1, 20.0, 300)]


def test_single_rank_reduction_is_identity():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max_sum(None, 12.5, 7, "cpu") == (12.5, 7)
