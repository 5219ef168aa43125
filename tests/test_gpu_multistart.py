"""Batched random-restart CP-ALS (one plan, restarts concatenated by
columns) against independent single runs with the same seeds."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden, rel_fro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("Re", [8, 16])
@pytest.mark.parametrize("layout,kernel,graphs", [("pingpong", "gs", True), ("ncopy", "gs", True),
                                                  ("pingpong", "gs", False),
                                                  ("ncopy", "jacobi", True)])
def test_restarts_follow_independent_runs(layout, kernel, graphs, Re):
    """Re = 16 takes the block-diagonal map on the FP64 tensor pipe, Re = 8
    the scalar one."""
    import dynasor_plus_b200 as d
    g = load_golden("ref_cpals_r5.npz")
    dims = g["dims"]
    idx = [g[f"idx{n}"] for n in range(len(dims))]
    K = 4
    iters = 3 if kernel == "jacobi" else 30
    tol = 0.0 if kernel == "jacobi" else 1e-4
    p = d.Plan(dims, g["vals"], idx, threads=int(g["T"]), rank=K * Re, layout=layout)
    batch = p.cpals_multistart(K, max_iters=iters, tol=tol, seed=42, kernel=kernel, graphs=graphs)
    Yb = [p.factor(n) for n in range(len(dims))]
    p.close()
    for k in range(K):
        q = d.Plan(dims, g["vals"], idx, threads=int(g["T"]), rank=Re, layout=layout)
        r = q.cpals(max_iters=iters, tol=tol, seed=42 + k, kernel=kernel)
        assert batch[k]["iters_done"] == r["iters_done"]
        # Jacobi iterations amplify rounding differences (see test_gpu_cpals)
        assert np.max(np.abs(batch[k]["fit_history"] - r["fit_history"])) < (
            1e-4 if kernel == "jacobi" else 1e-5)
        for n in range(len(dims)):
            assert rel_fro(Yb[n][:, k * Re:(k + 1) * Re], q.factor(n)[:, :Re]) < 1e-3
        q.close()


def test_restarts_reject_bad_rank_split():
    import dynasor_plus_b200 as d
    from dynasor_plus_b200._lib import DgpuError
    g = load_golden("ref_cpals_r5.npz")
    dims = g["dims"]
    idx = [g[f"idx{n}"] for n in range(len(dims))]
    p = d.Plan(dims, g["vals"], idx, threads=2, rank=30)
    with pytest.raises(DgpuError):
        p.cpals_multistart(4, max_iters=2)
    p.close()
