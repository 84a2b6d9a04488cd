"""The multi-GPU bench path runs independent replicas (no data-path
collective): each rank times its own run and the job's time is the maximum
over ranks.  Exercised here with world_size 2 on the gloo backend (CPU)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 10.0 * (rank + 1)                       # the two replicas took 10 ms and 20 ms
    ms_max = bench.max_over_ranks(ms, world, "cpu")
    out[rank] = (ms_max, bench.aggregate_rate(1_000_000, world, ms_max))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(2):
        ms_max, rate = res[r]
        assert ms_max == 20.0                     # max over ranks, identical on every rank
        assert rate == pytest.approx(2 * 1_000_000 / 20e-3 / 1e9)

