"""Owner-computes CP-ALS across ranks (dynasor_plus_b200.distributed): every
rank owns a contiguous, nonzero-balanced block of rows of every mode and
keeps only those rows' nonzeros; factors are rebuilt by all-gather, Grams
and column norms by all-reduce.  Here the ranks are gloo processes on the
CPU and each rank's MTTKRP rows come from the FP64 oracle (the GPU box of
these tests has one GPU; tests/test_gpu_owner_computes.py runs the engine's
MTTKRP through the same driver on it).  The run must follow the
single-process FP64 CP-ALS from the same initial factors."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _OracleRows:
    """A rank's MTTKRP rows in FP64 from the oracle, over the rank's own
    nonzeros of each mode."""

    def __init__(self, dims, vals, idx, blocks, me, R):
        from oracle import bindings as B
        self.B, self.dims, self.blocks, self.me, self.R = B, dims, blocks, me, R
        self.sub = []
        for n in range(len(dims)):
            lo, hi = blocks[n][me], blocks[n][me + 1]
            sel = np.flatnonzero((idx[n] >= lo) & (idx[n] < hi))
            self.sub.append((vals[sel], [i[sel] for i in idx]))

    def __call__(self, n, Y):
        import torch
        lo, hi = self.blocks[n][self.me], self.blocks[n][self.me + 1]
        v, ix = self.sub[n]
        out = self.B.mttkrp_f64(v, ix, n, [y.numpy() for y in Y], self.R, int(self.dims[n]))
        return torch.from_numpy(np.ascontiguousarray(out[lo:hi]))


def _case(name):
    from dynasor_plus_b200 import synth
    if name == "cp":
        return synth.cp_truth((300, 200, 100), 30_000, 4, 0.01, seed=11), 8, 20
    return synth.zipf((2000, 500, 120), draws=40_000, s=1.1, seed=13), 16, 6


def _rank_main(rank, ws, port, name, out):
    import datetime
    import torch.distributed as dist
    from dynasor_plus_b200 import distributed as D
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=120))
    try:
        (dims, vals, idx), R, it = _case(name)
        blocks = [D.row_blocks(np.bincount(idx[n], minlength=int(dims[n])), ws)
                  for n in range(len(dims))]
        rows = _OracleRows(dims, vals, idx, blocks, rank, R)
        run = D.OwnerComputesCpals(dims, vals, idx, R, group=None, device="cpu",
                                   local_mttkrp=rows)
        assert run.blocks == blocks
        r = run.run(max_iters=it, tol=0.0, seed=42)
        out.put((rank, r["fit_history"], [f[:, :R] for f in r["factors"]], r["lambda"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2, 3])
@pytest.mark.parametrize("name", ["cp", "zipf"])
def test_ranks_follow_single_process_fp64(bindings, ws, name):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, name, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(ws)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    (dims, vals, idx), R, it = _case(name)
    fit64, Y64, lam64 = bindings.cpals_f64(dims, vals, idx, R, it, 0.0, seed=42)
    for rank, fits, Y, lam in res:
        assert np.max(np.abs(fits - fit64)) < 1e-6, (rank, fits, fit64)
        for n in range(3):
            err = np.linalg.norm(Y[n] - Y64[n][:, :R]) / np.linalg.norm(Y64[n][:, :R])
            assert err < 1e-4, (rank, n, err)
    # every rank ends with the same factors
    for _, _, Y, _ in res[1:]:
        for n in range(3):
            assert np.array_equal(Y[n], res[0][2][n])


def test_row_blocks_balance_nonzeros():
    from dynasor_plus_b200 import distributed as D
    counts = np.array([5, 0, 0, 100, 1, 1, 1, 1, 40, 0])
    b = D.row_blocks(counts, 3)
    assert b[0] == 0 and b[-1] == len(counts) and all(x <= y for x, y in zip(b, b[1:]))
    assert b == [0, 4, 4, 10]          # row 3 holds 100 of the 149 nonzeros
    b = D.row_blocks(np.ones(9, np.int64), 3)
    assert b == [0, 3, 6, 9]
    b = D.row_blocks(np.zeros(5, np.int64), 2)
    assert b == [0, 2, 5]
    b = D.row_blocks(np.array([7]), 4)
    assert b[0] == 0 and b[-1] == 1
