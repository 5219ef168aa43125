"""The all-modes pass (dgpu_mttkrp_all_modes; spmttkrp_all_modes_dynasor,
src/dynasor.cpp:592-817, kernel.cpp:830-1039): every mode's MTTKRP from one
factor snapshot, in one pass over the live nonzeros, on every layout,
against FP64 MTTKRPs of each mode."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_fro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("layout", ["pingpong", "ncopy", "morton"])
@pytest.mark.parametrize("shape,draws,R", [((3000, 700, 200), 60_000, 16),
                                            ((400, 300, 60, 20), 50_000, 32),
                                            ((5000, 40, 30), 40_000, 48)])
def test_all_modes_pass_matches_fp64(bindings, layout, shape, draws, R):
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf(shape, draws=draws, s=1.1, seed=41)
    p = d.Plan(dims, vals, idx, threads=4, rank=R, layout=layout)
    Y = bindings.uniform_factors(3, dims, R)
    for n in range(len(dims)):
        p.set_factor(n, Y[n])
    if layout == "pingpong":
        p.process(0)                       # any slab order: the pass is order-free
    p.all_modes()
    for n in range(len(dims)):
        y64 = bindings.mttkrp_f64(vals, idx, n, Y, R, int(dims[n]))
        assert rel_fro(p.yhat(n)[:, :R], y64[:, :R]) < 1e-5, (layout, n)
    p.close()
