"""The multi-GPU path of bench.py is N independent replicas (the FLIP step does not shard): ranks
meet only at a barrier and the max-over-ranks reduction of their device times.  This runs that
host logic with world_size 2 over gloo on the CPU."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        bench.barrier(2)
        slowest = bench.max_over_ranks(2, 10.0 * (rank + 1))
        # value = units all ranks processed / the slowest rank's time
        units = 2 * 1000
        q.put((rank, slowest, units / slowest))
        bench.barrier(2)
    finally:
        dist.destroy_process_group()


def test_two_replicas_agree_on_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]
    assert all(abs(r[2] - 100.0) < 1e-12 for r in res)
