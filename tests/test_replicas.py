"""Multi-process replica logic of bench.py on CPU with the gloo backend
(world size 2): every rank agrees on the slowest rank's time, and the job
value counts all ranks' steps."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = bench.reduce_max(10.0 + 5.0 * rank, torch.device("cpu"), world)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ms))


def test_reduce_max_over_two_gloo_ranks():
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 15.0, 1: 15.0}


def test_reduce_max_single_process_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.reduce_max(3.5, torch.device("cpu"), 1) == 3.5
