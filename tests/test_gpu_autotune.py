"""dgpu_plan_autotune: chunk sizes, digit widths and the MTTKRP grid
target change no permutation -- a tuned plan's slab after the tuning sweeps
equals an untuned plan's after as many sweeps, bit for bit -- and results
only by FP32 summation order."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_fro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("layout", ["pingpong", "ncopy"])
def test_tuned_plan_keeps_the_permutation_and_results(bindings, layout):
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf((200_000, 40_000, 10_000), draws=3_000_000, s=1.1, seed=23)
    R = 16
    Y = bindings.uniform_factors(9, dims, R)
    tuned = d.Plan(dims, vals, idx, threads=8, rank=R, layout=layout)
    plain = d.Plan(dims, vals, idx, threads=8, rank=R, layout=layout)
    for n in range(3):
        tuned.set_factor(n, Y[n])
        plain.set_factor(n, Y[n])
    r = tuned.autotune(sweeps=1)
    print(f"\nautotune {layout}: {r}")
    assert r["candidates"] >= 3 and r["tuned_ms"] <= r["default_ms"] * 1.05
    for _ in range(2 * r["candidates"]):          # one warm-up + one timed sweep each
        plain.sweep()
    for n in range(3):
        tuned.process(n)
        plain.process(n)
        gv, gi = tuned.slab()
        pv, pi = plain.slab()
        assert np.array_equal(gv, pv) and all(np.array_equal(a, b) for a, b in zip(gi, pi)), n
        assert rel_fro(tuned.yhat(n)[:, :R], plain.yhat(n)[:, :R]) < 1e-5
    fit = tuned.cpals(max_iters=5, tol=0.0, seed=42)["fit_history"]
    fit64, _, _ = bindings.cpals_f64(dims, vals, idx, R, 5, 0.0, seed=42)
    assert np.max(np.abs(fit - fit64)) < 1e-6
    tuned.close()
    plain.close()


def test_autotune_rejects_a_plan_between_modes():
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((300, 200, 100), 20_000, seed=4)
    p = d.Plan(dims, vals, idx, threads=4, rank=8)
    p.process(0)
    with pytest.raises(d.DgpuError) as e:
        p.autotune()
    assert e.value.code == -6
    p.close()
