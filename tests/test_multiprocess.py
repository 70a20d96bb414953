"""World-size-2 gloo check of the multi-replica reduction bench.py uses: each
rank times its own replica; rank 0 reports total fields over the slowest rank's
time."""
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [120.0, 150.0][rank]
    fields = 40
    t = torch.tensor([ms], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    value = fields * world / (float(t[0]) / 1000.0)
    dist.barrier()
    if rank == 0:
        q.put(value)
    dist.destroy_process_group()


def test_replica_throughput_uses_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert abs(q.get(timeout=5) - 80 / 0.150) < 1e-6
