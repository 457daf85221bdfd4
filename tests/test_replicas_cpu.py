"""The multi-GPU bench path runs independent replicas (the reconstruction does
not shard): its only cross-rank steps are the barriers around the timed region
and the max over ranks of the device times.  Here two gloo ranks on the CPU
exercise exactly those helpers of bench.py."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        bench.barrier(ws)
        # rank r reports (r + 1) * 1.5 seconds: every rank must see the slowest
        v = bench.max_over_ranks((rank + 1) * 1.5, ws, torch.device("cpu"))
        bench.barrier(ws)
        out[rank] = v
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_barrier_two_gloo_ranks():
    ws = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, out)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert dict(out) == {0: 3.0, 1: 3.0}


def test_single_rank_needs_no_process_group():
    import bench
    assert not dist.is_initialized()
    bench.barrier(1)
    assert bench.max_over_ranks(2.5, 1, torch.device("cpu")) == 2.5
