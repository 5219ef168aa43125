"""Owner-computes CP-ALS with the engine's MTTKRP on the GPU
(dynasor_plus_b200.distributed).  One GPU is available, so: (1) a single
rank, with and without an NCCL process group, follows FP64 CP-ALS and the
single-plan run; (2) the row blocks of two ranks are built as two sets of
engine plans in one process, and their MTTKRP rows, put together, equal the
FP64 MTTKRP of the whole tensor; (3) two ranks run as two processes on this
GPU, each with its own engine plans, over a gloo group (collectives staged
through host memory), and follow FP64 CP-ALS."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from conftest import rel_fro

pytestmark = pytest.mark.gpu


def _case():
    from dynasor_plus_b200 import synth
    return synth.cp_truth((3000, 2000, 100), 300_000, 4, 0.01, seed=11)


@pytest.mark.parametrize("group", [False, True])
def test_single_rank_follows_fp64_and_the_plan(bindings, group):
    import torch
    import torch.distributed as dist
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import distributed as D
    dims, vals, idx = _case()
    R, it = 8, 12
    if group:
        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            port = s.getsockname()[1]
        os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
        import datetime
        dist.init_process_group("nccl", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=60),
                                device_id=torch.device("cuda", 0))
    try:
        run = D.OwnerComputesCpals(dims, vals, idx, R, threads=8)
        r = run.run(max_iters=it, tol=0.0, seed=42)
        run.close()
    finally:
        if group:
            dist.destroy_process_group()
    fit64, Y64, _ = bindings.cpals_f64(dims, vals, idx, R, it, 0.0, seed=42)
    p = d.Plan(dims, vals, idx, threads=8, rank=R)
    rp = p.cpals(max_iters=it, tol=0.0, seed=42)
    p.close()
    print(f"\nowner-computes, 1 rank: max |fit - fp64| {np.max(np.abs(r['fit_history'] - fit64)):.2e}, "
          f"vs plan {np.max(np.abs(r['fit_history'] - rp['fit_history'])):.2e}")
    assert np.max(np.abs(r["fit_history"] - fit64)) < 1e-6
    assert np.max(np.abs(r["fit_history"] - rp["fit_history"])) < 1e-6
    for n in range(3):
        assert rel_fro(r["factors"][n][:, :R], Y64[n][:, :R]) < 1e-4


def test_two_ranks_engine_rows_cover_the_mttkrp(bindings):
    import torch
    from dynasor_plus_b200 import distributed as D
    dims, vals, idx = _case()
    R, ws = 8, 2
    blocks = [D.row_blocks(np.bincount(idx[n], minlength=int(dims[n])), ws) for n in range(3)]
    dev = torch.device("cuda", 0)
    ranks = [D.EngineMttkrp(dims, vals, idx, blocks, me, R, 8, dev) for me in range(ws)]
    Y = [torch.from_numpy(bindings.uniform_factors(5, dims, R)[n]).to(dev) for n in range(3)]
    Yh = [y.cpu().numpy() for y in Y]
    for n in range(3):
        rows = torch.cat([ranks[me](n, Y) for me in range(ws)]).cpu().numpy()
        y64 = bindings.mttkrp_f64(vals, idx, n, Yh, R, int(dims[n]))
        assert rows.shape[0] == int(dims[n])
        assert rel_fro(rows[:, :R], y64[:, :R]) < 1e-5, n
    for r in ranks:
        r.close()


def _proc_rank(rank, ws, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    from dynasor_plus_b200 import distributed as D
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=120))
    try:
        dims, vals, idx = _case()
        run = D.OwnerComputesCpals(dims, vals, idx, 8, threads=8, device="cuda:0")
        assert run.stage
        r = run.run(max_iters=12, tol=0.0, seed=42)
        run.close()
        out.put((rank, r["fit_history"], [f[:, :8] for f in r["factors"]]))
    finally:
        dist.destroy_process_group()


def test_two_processes_follow_fp64(bindings):
    """Two ranks as two processes, each with its own engine plans on this
    GPU and its own CUDA context; the collectives are gloo's, staged through
    host memory (no kernel of one rank waits for the other's)."""
    import torch.multiprocessing as mp
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_proc_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(ws)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    dims, vals, idx = _case()
    fit64, Y64, _ = bindings.cpals_f64(dims, vals, idx, 8, 12, 0.0, seed=42)
    for rank, fits, Y in res:
        print(f"\nowner-computes, 2 processes, rank {rank}: max |fit - fp64| "
              f"{np.max(np.abs(fits - fit64)):.2e}")
        assert np.max(np.abs(fits - fit64)) < 1e-6
        for n in range(3):
            assert rel_fro(Y[n], Y64[n][:, :8]) < 1e-4, (rank, n)
    for n in range(3):
        assert np.array_equal(res[0][2][n], res[1][2][n])
