"""Multi-GPU path of bench.py on CPU: independent replicas, one per rank,
with the step time reduced as the max over ranks (world size 2, gloo)."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    t = [3.5, 7.25][rank]
    m = bench.reduce_max(t)
    out.put((rank, m))
    dist.barrier()
    dist.destroy_process_group()


def test_reduce_max_over_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    assert res == {0: 7.25, 1: 7.25}


def test_reduce_max_single_process_is_identity():
    import bench
    assert bench.reduce_max(1.5) == 1.5
