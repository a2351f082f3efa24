"""The multi-rank path of bench.py on CPU: two gloo ranks (world size 2),
barrier and max-over-ranks of per-replica device times, as `bench.py --gpus N`
uses them with NCCL.  The hot path itself does not shard (replicas only)."""

from __future__ import annotations

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


def _worker(rank, ws, port, out):
    import sys
    from datetime import timedelta
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["RANK"] = str(rank)
    os.environ["WORLD_SIZE"] = str(ws)
    os.environ["LOCAL_RANK"] = str(rank)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    try:
        assert bench._dist() == (ws, rank, rank)
        bench._barrier(ws)
        t = 10.0 + 5.0 * rank          # this replica's "device time"
        out[rank] = bench._max_over_ranks(t, ws)
        bench._barrier(ws)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_max():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("gloo rank did not finish")
        assert p.exitcode == 0
    assert out[0] == out[1] == 15.0
