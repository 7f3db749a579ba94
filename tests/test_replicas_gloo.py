"""The multi-GPU path of bench.py runs independent replicas whose only
collective is the max-over-ranks reduction of the measured time.  Checked here
with two gloo ranks on the CPU (no GPU needed)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, values, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks(values[rank], dist, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    values = [3.25, 7.5]
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, values, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 7.5


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks(1.5, None) == 1.5
