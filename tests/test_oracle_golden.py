"""Pin the oracle (this project's CPU restatement) against golden fixtures
produced by the reference itself (tests/golden/make_golden.py).  CPU only."""
from __future__ import annotations

import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden, rel_fro

SWEEP_CASES = sorted(os.path.basename(p) for p in glob.glob(os.path.join(GOLDEN, "ref_*.npz"))
                     if "cpals" not in p)


def _case(g):
    dims = g["dims"]
    N = len(dims)
    return dims, g["vals"], [g[f"idx{n}"] for n in range(N)], int(g["T"]), int(g["R"]), \
        bool(int(g["fiber"]))


@pytest.mark.parametrize("name", SWEEP_CASES)
def test_plan_tables_match_reference(bindings, name):
    g = load_golden(name)
    dims, vals, idx, T, R, fiber = _case(g)
    o = bindings.Oracle(dims, vals, idx, T)
    assert np.array_equal(o.shift, g["shift"])
    assert np.array_equal(o.K, g["K"])
    assert np.array_equal(o.kclass, g["kclass"])
    for n in range(len(dims)):
        b, e = o.shards(n)
        assert np.array_equal(b, g[f"sbeg{n}"]) and np.array_equal(e, g[f"send{n}"])
        c, f = o.schedule(n)
        assert np.array_equal(c, g[f"sched_counts{n}"]) and np.array_equal(f, g[f"sched{n}"])
        assert np.array_equal(o.cursors(n), g[f"cursors{n}"])
    v, ix = o.slab()
    assert np.array_equal(v, g["slab0_v"])
    for n in range(len(dims)):
        assert np.array_equal(ix[n], g[f"slab0_i{n}"])


@pytest.mark.parametrize("name", SWEEP_CASES)
def test_remap_and_fp32_fold_match_reference(bindings, name):
    """Slab after every process(n) is bit-identical; the FP32 fold in slab
    order reproduces the reference kernel's Yhat bit for bit."""
    g = load_golden(name)
    dims, vals, idx, T, R, fiber = _case(g)
    N = len(dims)
    o = bindings.Oracle(dims, vals, idx, T)
    Y = [g[f"Y{n}"] for n in range(N)]
    sweeps = len([k for k in g if k.startswith("yhat_s") and k.endswith("_m0")])
    for s in range(sweeps):
        for n in range(N):
            if fiber and o.kclass[n] == 2:
                o.fiber_sort(n)
            v, ix = o.slab()
            yf = bindings.mttkrp_f32_fold(v, ix, n, Y, int(dims[n]))
            assert np.array_equal(yf, g[f"yhat_s{s}_m{n}"]), (s, n)
            o.remap(n)
            v, ix = o.slab()
            assert np.array_equal(v, g[f"slab_s{s}_m{n}_v"]), (s, n)
            for k in range(N):
                assert np.array_equal(ix[k], g[f"slab_s{s}_m{n}_i{k}"]), (s, n, k)


@pytest.mark.parametrize("name", SWEEP_CASES)
def test_fp64_mttkrp_vs_reference_oracle(bindings, name):
    g = load_golden(name)
    dims, vals, idx, T, R, fiber = _case(g)
    N = len(dims)
    Y = [g[f"Y{n}"] for n in range(N)]
    for n in range(N):
        y64 = bindings.mttkrp_f64(vals, idx, n, Y, R, int(dims[n]))
        assert rel_fro(g[f"yref{n}"][:, :R], y64[:, :R]) < 1e-6


def test_uniform_init_matches_reference_inputs(bindings):
    g = load_golden("ref_3d7_T2_R16.npz")
    Y = bindings.uniform_factors(42, g["dims"], int(g["R"]))
    for n in range(len(g["dims"])):
        assert np.array_equal(Y[n], g[f"Y{n}"])


def test_cpals_fp64_oracle_tracks_reference(bindings):
    g = load_golden("ref_cpals_r5.npz")
    dims = g["dims"]
    idx = [g[f"idx{n}"] for n in range(len(dims))]
    fit, Y, lam = bindings.cpals_f64(dims, g["vals"], idx, int(g["R"]), int(g["iters"]),
                                     float(g["tol"]), seed=42)
    ref = g["fit"]
    assert len(fit) == len(ref)
    # the reference truncates <T,M> to FP32 (src/dynasor_linalg.cpp:365); on
    # this well-conditioned rank-5 problem that stays below 1e-4
    assert np.max(np.abs(fit - ref)) < 1e-4
