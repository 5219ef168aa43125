"""Owner-computes CP-ALS with the engine's MTTKRP on the GPU
(dynasor_plus_b200.distributed).  One GPU is available, so: (1) a single
rank, with and without an NCCL process group, follows FP64 CP-ALS and the
single-plan run; (2) the row blocks of two ranks are built as two sets of
engine plans in one process, and their MTTKRP rows, put together, equal the
FP64 MTTKRP of the whole tensor (the collectives themselves run on gloo
ranks in tests/test_owner_computes_gloo.py)."""
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
