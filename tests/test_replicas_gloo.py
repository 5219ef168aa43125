"""bench.py on N GPUs runs N independent replicas (no collective on the data
path): the job time is the slowest rank's, the job value is N x nnz per
step over it.  The reduction and the value arithmetic run here as two gloo
ranks on the CPU (the GPU box of these tests has one GPU)."""
from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    import torch.distributed as dist
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        got_ws, got_rank, got_local = bench.dist_setup()
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, got_ws, device="cpu")
        dist.barrier()
        out.put((got_rank, got_ws, got_local, ms, bench.job_gnnz_s(1_000_000, got_ws, ms)))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank_and_sum_the_work():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, (got_rank, ws, local, ms, value) in enumerate(res):
        assert (got_rank, ws, local) == (rank, 2, rank)
        assert ms == pytest.approx(15.0)              # rank 1 is the slower one
        assert value == pytest.approx(2 * 1_000_000 / 15e-3 / 1e9)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_gnnz_s(2_000_000, 1, 2.0) == pytest.approx(1.0)
