"""Kept partition offset tables of the PingPong sweep.

After one full cycle of modes the slab's arrangement is a function of the
coordinates alone (each mode's shard and row key plus the schedule order
break every tie), so the partition passes of every later sweep reuse the
per-(chunk, bucket) offsets computed in the first such sweep -- the
reference builds its remap cursor table once as well
(src/dynasor_preprocess.cpp:439-462).  The slabs are compared with the
oracle's remap and fiber sort over several sweeps with the tables kept, with
the device check mode (every kept table recomputed and compared: a
difference raises), and against a plan that recomputes every table."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_fro

pytestmark = pytest.mark.gpu

CASES = {
    # Zipf rows: shards larger than one tile and one fiber chunk, so chunk
    # boundaries fall inside shards (counts depend on the arrangement)
    "zipf3": ((20000, 3000, 500), 400000, 16, 16, 3, "zipf"),
    "uniform4": ((300, 200, 100, 50), 200000, 8, 16, 4, "uniform"),
    # more next-mode shards than one pass handles: multi-pass remaps
    "lsd": ((70000, 50000, 3000), 60000, 2048, 16, 21, "uniform"),
}


def _tensor(kind, dims, nnz, seed):
    from dynasor_plus_b200 import synth
    if kind == "zipf":
        return synth.zipf(dims, draws=nnz, s=1.1, seed=seed)
    return synth.uniform(dims, nnz, seed=seed)


def _slab_equal(p, o):
    v, ix = o.slab()
    pv, pix = p.slab()
    return np.array_equal(pv, v) and all(np.array_equal(a, b) for a, b in zip(pix, ix))


@pytest.mark.parametrize("replay", ["1", "0"])
@pytest.mark.parametrize("digit", ["8", "2"])
@pytest.mark.parametrize("fiber", [True, False])
@pytest.mark.parametrize("case", sorted(CASES))
def test_sweeps_with_kept_tables_match_oracle(bindings, monkeypatch, case, fiber, digit, replay):
    """Four sweeps with the kept tables checked on the device: every slab
    equals the oracle's, with the passes replayed from their recordings
    (replay "1", the default) or ranked on the kept tables ("0").  Digit
    width 2 gives fiber sorts of more LSD passes than the tables kept per
    sort (the later passes recompute)."""
    import dynasor_plus_b200 as d
    dims, nnz, T, R, seed, kind = CASES[case]
    monkeypatch.setenv("DGPU_PART_CACHE_CHECK", "1")
    monkeypatch.setenv("DGPU_FIBER_DIGIT_BITS", digit)
    monkeypatch.setenv("DGPU_PART_REPLAY", replay)
    dims, vals, idx = _tensor(kind, dims, nnz, seed)
    N = len(dims)
    o = bindings.Oracle(dims, vals, idx, T)
    p = d.Plan(dims, vals, idx, threads=T, rank=R, fiber=fiber)
    Y = bindings.uniform_factors(seed, dims, R)
    for n in range(N):
        p.set_factor(n, Y[n])
    for s in range(4):
        for n in range(N):
            if fiber and o.kclass[n] == 2:
                o.fiber_sort(n)
            if s == 3:
                v, ix = o.slab()
                y64 = bindings.mttkrp_f64(v, ix, n, Y, R, int(dims[n]))
            o.remap(n)
            p.process(n)
            assert _slab_equal(p, o), f"sweep {s} mode {n}"
            if s == 3:
                assert rel_fro(p.yhat(n)[:, :R], y64[:, :R]) <= 1e-5, n
    p.close()


def test_kept_tables_equal_recomputed_cpals(monkeypatch):
    """CP-ALS from a fresh PingPong plan (its first iteration is the slab's
    first cycle, the second fills the kept tables, the device loop runs on
    them) against a plan that recomputes every table: same slab after the
    run, same fits up to the MTTKRP's atomic summation order."""
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf((20000, 3000, 500), draws=400000, s=1.1, seed=8)
    runs = []
    for cache in ("1", "0"):
        monkeypatch.setenv("DGPU_PART_CACHE", cache)
        monkeypatch.setenv("DGPU_PART_CACHE_CHECK", cache)
        p = d.Plan(dims, vals, idx, threads=16, rank=16)
        r1 = p.cpals(max_iters=12, tol=0.0, seed=42)
        r2 = p.cpals(max_iters=12, tol=0.0, seed=42)       # the kept loop graph
        runs.append((r1, r2, p.slab()))
        p.close()
    (a1, a2, sa), (b1, b2, sb) = runs
    assert a1["iters_done"] == b1["iters_done"] == 12
    for x, y in ((a1, b1), (a2, b2), (a1, a2)):
        assert np.allclose(x["fit_history"], y["fit_history"], rtol=0, atol=1e-7)
    assert np.array_equal(sa[0], sb[0]) and all(np.array_equal(u, v) for u, v in zip(sa[1], sb[1]))


def test_kept_tables_follow_autotuned_knobs(bindings):
    """Autotuning rebuilds the partition lists and changes digit widths:
    the kept tables are dropped with them, and sweeps after it still equal
    the oracle's."""
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf((20000, 3000, 500), draws=300000, s=1.1, seed=9)
    T, R = 16, 16
    o = bindings.Oracle(dims, vals, idx, T)
    p = d.Plan(dims, vals, idx, threads=T, rank=R)
    Y = bindings.uniform_factors(9, dims, R)
    for n in range(3):
        p.set_factor(n, Y[n])

    def sweep():
        for n in range(3):
            if o.kclass[n] == 2:
                o.fiber_sort(n)
            o.remap(n)
            p.process(n)
            assert _slab_equal(p, o), n

    sweep()
    sweep()
    # the tuning sweeps advance the slab; past its first cycle a sweep
    # leaves the arrangement where it was, so it still equals the oracle's
    p.autotune(sweeps=1)
    assert _slab_equal(p, o)
    sweep()
    sweep()
    p.close()


@pytest.mark.parametrize("ctas", ["1", "3"])
@pytest.mark.parametrize("case", ["zipf3", "lsd"])
def test_remap_first_overlap_matches_oracle(bindings, monkeypatch, case, ctas):
    """DGPU_OVERLAP=2: each mode's first remap pass (replayed from the third
    sweep on, at most `ctas` CTAs per SM) is launched before the MTTKRP on
    the second stream, and a later LSD pass of the remap waits for the
    MTTKRP; the slabs equal the oracle's and Yhat its FP64 MTTKRP."""
    import dynasor_plus_b200 as d
    dims, nnz, T, R, seed, kind = CASES[case]
    monkeypatch.setenv("DGPU_OVERLAP", "2")
    monkeypatch.setenv("DGPU_REMAP_CTAS", ctas)
    dims, vals, idx = _tensor(kind, dims, nnz, seed)
    o = bindings.Oracle(dims, vals, idx, T)
    p = d.Plan(dims, vals, idx, threads=T, rank=R)
    Y = bindings.uniform_factors(seed, dims, R)
    for n in range(3):
        p.set_factor(n, Y[n])
    for s in range(4):
        for n in range(3):
            if o.kclass[n] == 2:
                o.fiber_sort(n)
            v, ix = o.slab()
            y64 = bindings.mttkrp_f64(v, ix, n, Y, R, int(dims[n]))
            o.remap(n)
            p.process(n)
            assert _slab_equal(p, o), f"sweep {s} mode {n}"
            assert rel_fro(p.yhat(n)[:, :R], y64[:, :R]) <= 1e-5, (s, n)
    p.close()

