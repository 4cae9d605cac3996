"""The multi-rank host logic on CPU: two gloo ranks (127.0.0.1) share specimens and time
reductions exactly as NCCL ranks on GPUs do (pdcuda/replicas.py). No GPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from pdcuda.replicas import partition_specimens, throughput, reduce_max


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = partition_specimens(sizes, world)[rank]
        units = sum(sizes[k] for k in mine)
        seconds = 1.0 + rank  # rank 1 is the slower one
        rate = throughput(units, seconds, dist)
        tmax = reduce_max(seconds, dist)
        dist.barrier()
        q.put((rank, mine, units, rate, tmax))
    finally:
        dist.destroy_process_group()


def test_partition_balances_and_covers():
    sizes = [200_000, 20_000, 150_000, 90_000, 60_000, 110_000, 30_000]
    parts = partition_specimens(sizes, 3)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[k] for k in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)
    assert partition_specimens(sizes, 1) == [list(range(len(sizes)))]
    # deterministic
    assert parts == partition_specimens(sizes, 3)


@pytest.mark.timeout(120)
def test_two_gloo_ranks_share_specimens_and_time():
    sizes = [120_000, 80_000, 60_000, 40_000, 20_000]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in range(2))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    owned = sorted(k for _, mine, *_ in res for k in mine)
    assert owned == list(range(len(sizes)))
    total = sum(sizes)
    for rank, mine, units, rate, tmax in res:
        assert tmax == 2.0                      # max over ranks
        assert rate == pytest.approx(total / 2.0)  # all units over the slowest rank's time
