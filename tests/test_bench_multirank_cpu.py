"""The N > 1 path of bench.py without a GPU: two gloo ranks on 127.0.0.1
(independent replicas, one process each) check the rank environment, the
slowest-rank reduction behind the timed and end-to-end figures, the whole-job
throughput and that the reference arm runs on rank 0 only."""

import contextlib
import io
import os
import socket
import sys
from datetime import timedelta

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import argparse

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    try:
        out = {"dist": bench._dist()}
        out["t_max"] = bench.max_over_ranks(1.5 + rank, ws, device="cpu")   # rank 1 is the slow one
        out["value"] = bench.replica_throughput(ws, 12 * 3, out["t_max"])
        if rank != 0:  # the reference arm does no work and prints nothing off rank 0
            buf = io.StringIO()
            args = argparse.Namespace(workload="checkerboard24", steps=1, warmup=0, gpus=ws)
            with contextlib.redirect_stdout(buf):
                bench.run_reference(args)
            out["reference_stdout"] = buf.getvalue()
        dist.barrier()
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    try:
        for _ in range(2):
            rank, out = q.get(timeout=240)
            res[rank] = out
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    for rank in (0, 1):
        assert res[rank]["dist"] == (2, rank, rank)
        assert res[rank]["t_max"] == 2.5                        # the max over ranks, on every rank
        assert res[rank]["value"] == pytest.approx(2 * 36 / 2.5)  # all units over the slowest time
    assert res[1]["reference_stdout"] == ""


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.0, 1) == 3.0
    assert bench.replica_throughput(1, 36, 2.0) == 18.0
