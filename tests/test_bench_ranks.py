"""CPU test of the multi-process timing path of bench.py: two gloo ranks (one process per
rank, as torchrun launches them), each with its own step time; every rank must see the
maximum, which is the time the whole job took."""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(REPO))
    from bench import max_over_ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = max_over_ranks(10.0 + 5.0 * rank, dist, torch.device("cpu"))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_processes() -> None:
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs)
        assert dict(out) == {0: 15.0, 1: 15.0}


def test_max_over_ranks_single_process() -> None:
    sys.path.insert(0, str(REPO))
    from bench import max_over_ranks

    assert max_over_ranks(3.5, None, None) == 3.5
