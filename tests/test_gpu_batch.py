"""Several tensors decomposed in one batch (parallel device loops of one
graph launch) against the same runs one by one."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_fro

pytestmark = pytest.mark.gpu


def _tensors():
    from dynasor_plus_b200 import synth
    shapes = [((300, 200, 100), 30_000), ((1500, 90, 400), 120_000), ((60, 70, 80), 8_000),
              ((5000, 3000, 40), 250_000)]
    return [synth.cp_truth(d, nnz, 4, 0.01, seed=11 + i) for i, (d, nnz) in enumerate(shapes)]


@pytest.mark.parametrize("layout", ["ncopy", "pingpong"])
def test_batch_matches_single_runs(layout):
    import dynasor_plus_b200 as d
    ts = _tensors()
    plans = [d.Plan(dims, v, i, threads=8, rank=8, layout=layout) for dims, v, i in ts]
    batch = d.cpals_batch(plans, max_iters=40, tol=1e-4, seed=42)
    facs = [[p.factor(n) for n in range(3)] for p in plans]
    for p in plans:
        p.close()
    for k, (dims, v, i) in enumerate(ts):
        q = d.Plan(dims, v, i, threads=8, rank=8, layout=layout)
        r = q.cpals(max_iters=40, tol=1e-4, seed=42)
        assert batch[k]["iters_done"] == r["iters_done"]
        assert np.max(np.abs(batch[k]["fit_history"] - r["fit_history"])) < 1e-6
        for n in range(3):
            assert rel_fro(facs[k][n], q.factor(n)) < 1e-4
        q.close()


def test_batch_rejects_repeated_plan():
    import dynasor_plus_b200 as d
    from dynasor_plus_b200._lib import DgpuError
    dims, v, i = _tensors()[0]
    p = d.Plan(dims, v, i, threads=4, rank=8)
    with pytest.raises(DgpuError):
        d.cpals_batch([p, p], max_iters=2)
    p.close()


@pytest.mark.parametrize("layout,precision", [("ncopy", "fp32"), ("pingpong", "fp32"),
                                              ("ncopy", "bf16")])
def test_repeated_batch_reuses_its_loop_graph(layout, precision):
    """The batch's loop graph is kept on its first plan: a second call with
    the same options runs every iteration, the first included, in it; a call
    with other options captures a new one; every call equals single runs."""
    import dynasor_plus_b200 as d
    ts = _tensors()
    plans = [d.Plan(dims, v, i, threads=8, rank=8, layout=layout, precision=precision)
             for dims, v, i in ts]
    want = {}
    for tol in (1e-4, 1e-3):
        want[tol] = []
        for dims, v, i in ts:
            q = d.Plan(dims, v, i, threads=8, rank=8, layout=layout, precision=precision)
            want[tol].append(q.cpals(max_iters=40, tol=tol, seed=42))
            q.close()
    # BF16: rounding flips of gathered entries drift the fits by ~1e-6, which
    # can move a stop at |dfit| < tol by one iteration
    for tol in (1e-4, 1e-4, 1e-3, 1e-4, 1e-4):
        got = d.cpals_batch(plans, max_iters=40, tol=tol, seed=42)
        for k, r in enumerate(want[tol]):
            h, w = got[k]["fit_history"], r["fit_history"]
            if precision == "fp32":
                assert got[k]["iters_done"] == r["iters_done"], (tol, k)
                assert np.max(np.abs(h - w)) < 1e-6, (tol, k)
            else:
                assert abs(got[k]["iters_done"] - r["iters_done"]) <= 1, (tol, k)
                m = min(len(h), len(w))
                assert abs(h[0] - w[0]) < 1e-7, (tol, k)
                assert np.max(np.abs(h[:m] - w[:m])) < 1e-5, (tol, k)
    for p in plans:
        p.close()
