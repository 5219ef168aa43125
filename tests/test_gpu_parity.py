"""Parity of the CUDA path (through the C-ABI) with the reference and the
oracle.  Integer work (plan tables, remap permutation, fiber sort, NCopy
copies) must be bit-exact; MTTKRP values must be within relative Frobenius
1e-5 of the reference's FP32 result and of the FP64 oracle."""
from __future__ import annotations

import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden, rel_fro

pytestmark = pytest.mark.gpu

SWEEP_CASES = sorted(os.path.basename(p) for p in glob.glob(os.path.join(GOLDEN, "ref_*.npz"))
                     if "cpals" not in p)
TOL_FP32 = 1e-5          # bound vs the reference MTTKRP (FP32)
TOL_BF16 = 2e-2          # BF16 gathers (8-bit mantissa) vs FP64


def _plan(dims, vals, idx, T, R, **kw):
    import dynasor_plus_b200 as d
    return d.Plan(dims, vals, idx, threads=T, rank=R, **kw)


def _assert_slab(p, v_ref, i_ref, what):
    v, ix = p.slab()
    assert np.array_equal(v, v_ref), what
    for k in range(len(ix)):
        assert np.array_equal(ix[k], i_ref[k]), (what, k)


@pytest.mark.parametrize("overlap", ["1", "0", "2"])
@pytest.mark.parametrize("name", SWEEP_CASES)
def test_golden_sweeps(name, overlap, monkeypatch):
    # overlap "1": each PingPong MTTKRP runs on a second stream beside the
    # remap (the default); "0": both on the plan stream, one after the other;
    # "2": the remap's first pass launched first, the MTTKRP beside it
    monkeypatch.setenv("DGPU_OVERLAP", overlap)
    g = load_golden(name)
    dims = g["dims"]
    N = len(dims)
    idx = [g[f"idx{n}"] for n in range(N)]
    T, R, fiber = int(g["T"]), int(g["R"]), bool(int(g["fiber"]))
    p = _plan(dims, g["vals"], idx, T, R, fiber=fiber)
    inf = p.info()
    assert inf["mn_shift"] == list(g["shift"]) and inf["shards_per_mode"] == list(g["K"])
    assert inf["kernel_class"] == list(g["kclass"])
    for n in range(N):
        b, e = p.shards(n)
        assert np.array_equal(b, g[f"sbeg{n}"]) and np.array_equal(e, g[f"send{n}"])
        c, f = p.schedule(n)
        assert np.array_equal(c, g[f"sched_counts{n}"]) and np.array_equal(f, g[f"sched{n}"])
    _assert_slab(p, g["slab0_v"], [g[f"slab0_i{n}"] for n in range(N)], "after build")
    for n in range(N):
        p.set_factor(n, g[f"Y{n}"])
    sweeps = len([k for k in g if k.startswith("yhat_s") and k.endswith("_m0")])
    for s in range(sweeps):
        for n in range(N):
            p.process(n)
            y = p.yhat(n)
            assert rel_fro(y[:, :R], g[f"yhat_s{s}_m{n}"][:, :R]) <= TOL_FP32, (s, n)
            assert np.all(y[:, R:] == 0)
            _assert_slab(p, g[f"slab_s{s}_m{n}_v"], [g[f"slab_s{s}_m{n}_i{k}"] for k in range(N)],
                         f"sweep {s} mode {n}")


CASES = [
    # dims, nnz, T, R, seed
    ((37, 23, 11), 700, 1, 5, 1),
    ((37, 23, 11), 700, 3, 16, 2),
    ((200, 150, 90), 20000, 8, 32, 3),
    ((64, 32, 16, 8), 5000, 5, 48, 4),
    ((50, 40, 30, 20, 10), 6000, 2, 8, 5),
    ((300, 400), 8000, 4, 64, 6),           # N = 2
    ((5, 7, 3), 40, 64, 16, 7),             # threads >= mode sizes -> m_n = 1
    ((1, 9, 4), 30, 2, 3, 8),               # a mode of size 1
]


@pytest.mark.parametrize("fiber", [True, False])
@pytest.mark.parametrize("dims,nnz,T,R,seed", CASES)
def test_random_vs_oracle(bindings, dims, nnz, T, R, seed, fiber):
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform(dims, nnz, seed=seed)     # duplicates kept
    N = len(dims)
    o = bindings.Oracle(dims, vals, idx, T)
    p = _plan(dims, vals, idx, T, R, fiber=fiber)
    v, ix = o.slab()
    _assert_slab(p, v, ix, "after build")
    Y = bindings.uniform_factors(seed, dims, R)
    for n in range(N):
        p.set_factor(n, Y[n])
    for s in range(2):
        for n in range(N):
            if fiber and o.kclass[n] == 2:
                o.fiber_sort(n)
            v, ix = o.slab()
            y64 = bindings.mttkrp_f64(v, ix, n, Y, R, int(dims[n]))
            yf = bindings.mttkrp_f32_fold(v, ix, n, Y, int(dims[n]))
            o.remap(n)
            p.process(n)
            y = p.yhat(n)
            assert rel_fro(y[:, :R], y64[:, :R]) <= TOL_FP32, (s, n)
            assert rel_fro(y[:, :R], yf[:, :R]) <= TOL_FP32, (s, n)
            v, ix = o.slab()
            _assert_slab(p, v, ix, f"sweep {s} mode {n}")


def test_many_shards_lsd_path(bindings):
    """More next-mode shards than one partition pass handles (K > 2048):
    the remap runs as least-significant-digit passes and must still equal
    the one-pass stable counting sort."""
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((70000, 50000, 3000), 60000, seed=21)
    T = 2048
    o = bindings.Oracle(dims, vals, idx, T)
    assert o.K[0] > 2048 and o.K[1] > 2048
    p = _plan(dims, vals, idx, T, 16, fiber=True)
    v, ix = o.slab()
    _assert_slab(p, v, ix, "after build")
    Y = bindings.uniform_factors(3, dims, 16)
    for n in range(3):
        p.set_factor(n, Y[n])
    for n in range(3):
        if o.kclass[n] == 2:
            o.fiber_sort(n)
        v, ix = o.slab()
        y64 = bindings.mttkrp_f64(v, ix, n, Y, 16, int(dims[n]))
        o.remap(n)
        p.process(n)
        assert rel_fro(p.yhat(n)[:, :16], y64[:, :16]) <= TOL_FP32
        v, ix = o.slab()
        _assert_slab(p, v, ix, f"mode {n}")


def test_ncopy_copies_match_reference(refb):
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf((3000, 500, 200), draws=30000, s=1.1, seed=31)
    T, R = 4, 16
    ref = refb.Reference(dims, vals, idx)
    ref.build(T, "ncopy")
    p = _plan(dims, vals, idx, T, R, layout="ncopy", fiber=True)
    Y = refb.uniform_factors(9, dims, R)
    ref.factors(R)
    for n in range(3):
        v, ix, _ = ref.ncopy(n)
        pv, pix = p.copy(n)
        assert np.array_equal(pv, v) and all(np.array_equal(a, b) for a, b in zip(pix, ix)), n
        ref.set_Y(n, Y[n])
        p.set_factor(n, Y[n])
    ref.sweep_begin()
    for n in range(3):
        ref.process(n)
        p.process(n)
        assert rel_fro(p.yhat(n)[:, :R], ref.yhat(n)[:, :R]) <= TOL_FP32


def test_bf16_gathers_close_to_fp64(bindings):
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf((4000, 900, 300), draws=50000, s=1.1, seed=41)
    T, R = 8, 32
    o = bindings.Oracle(dims, vals, idx, T)
    p = _plan(dims, vals, idx, T, R, precision="bf16", fiber=False)
    Y = bindings.uniform_factors(5, dims, R)
    for n in range(3):
        p.set_factor(n, Y[n])
    for n in range(3):
        v, ix = o.slab()
        y64 = bindings.mttkrp_f64(v, ix, n, Y, R, int(dims[n]))
        o.remap(n)
        p.process(n)
        err = rel_fro(p.yhat(n)[:, :R], y64[:, :R])
        assert err <= TOL_BF16, (n, err)
        v, ix = o.slab()
        _assert_slab(p, v, ix, f"mode {n}")


def _round_bf16(y):
    """FP32 -> BF16 -> FP32 with round-to-nearest-even (finite inputs)."""
    b = np.ascontiguousarray(y, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("dims", [(4000, 900, 300), (3000, 700, 200, 60)])
@pytest.mark.parametrize("R", [16, 32, 48, 64, 128])
def test_bf16_rowrun_exact_on_rounded_factors(bindings, dims, R):
    """The row-run kernel with BF16 gathers (every lane-group shape, rank
    tiles at R = 128): FP32 products of the BF16-rounded factors, so it
    meets the FP32 bound against an FP64 MTTKRP of those rounded factors."""
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf(dims, draws=60000, s=1.1, seed=43 + R)
    N = len(dims)
    p = _plan(dims, vals, idx, 8, R, precision="bf16", accum="rowrun")
    rng = np.random.default_rng(R)
    Y = []
    for n in range(N):
        y = np.zeros((int(dims[n]), p.Rp), np.float32)
        y[:, :R] = rng.uniform(-1, 1, (int(dims[n]), R))
        Y.append(y)
        p.set_factor(n, y)
    Yb = [_round_bf16(y) for y in Y]
    for n in range(N):
        p.process(n)
        y64 = bindings.mttkrp_f64(vals, idx, n, Yb, R, int(dims[n]))
        got = p.yhat(n)
        assert rel_fro(got[:, :R], y64[:, :R]) <= TOL_FP32, (n, rel_fro(got[:, :R], y64[:, :R]))
        assert np.all(got[:, R:] == 0)
    p.close()


def test_out_of_order_mode_is_rejected():
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((20, 20, 20), 300, seed=1)
    p = _plan(dims, vals, idx, 2, 8)
    with pytest.raises(d.DgpuError) as e:
        p.process(1)
    assert e.value.code == -6


def test_bad_inputs_fail_loudly():
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((20, 20, 20), 300, seed=1)
    idx[1][5] = 20                      # out of range
    with pytest.raises(d.DgpuError) as e:
        _plan(dims, vals, idx, 2, 8)
    assert e.value.code == -5
    with pytest.raises(d.DgpuError) as e:
        _plan(dims, vals[:0], [i[:0] for i in idx], 2, 8)
    assert e.value.code == -4
    with pytest.raises(d.DgpuError):
        _plan(dims, vals, [i % 20 for i in idx], 0, 8)


def test_single_nonzero():
    import dynasor_plus_b200 as d
    dims = np.array([4, 5, 6], np.uint32)
    vals = np.array([2.5], np.float32)
    idx = [np.array([3], np.uint32), np.array([1], np.uint32), np.array([5], np.uint32)]
    p = d.Plan(dims, vals, idx, threads=2, rank=4)
    Y = [np.zeros((int(x), 16), np.float32) for x in dims]
    for n in range(3):
        Y[n][:, :4] = np.arange(1, 5) * (n + 1)
        p.set_factor(n, Y[n])
    p.process(0)
    y = p.yhat(0)
    expect = 2.5 * (np.arange(1, 5) * 2) * (np.arange(1, 5) * 3)
    assert np.allclose(y[3, :4], expect) and np.count_nonzero(y) == 4


@pytest.mark.parametrize("layout", ["pingpong", "ncopy"])
def test_host_sweep_overlapped_transfers_match_device_sweep(layout):
    """dgpu_mttkrp_sweep_host (uploads and downloads overlapping the mode
    passes) gives the Yhat of a plain device sweep, twice in a row, with
    pageable and pinned host buffers."""
    import torch
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf((3000, 800, 200), 300_000, 1.1, seed=4)
    R = 32
    rng = np.random.default_rng(3)
    Y = [rng.uniform(-1, 1, (int(dims[n]), R)).astype(np.float32) for n in range(3)]
    p = d.Plan(dims, vals, idx, threads=8, rank=R, layout=layout)
    Yp = [np.zeros((int(dims[n]), p.Rp), np.float32) for n in range(3)]
    for n in range(3):
        Yp[n][:, :R] = Y[n]
        p.set_factor(n, Yp[n])
    p.sweep()
    ref = [p.yhat(n) for n in range(3)]
    for pinned in (False, True, True):
        if pinned:
            Yin = [torch.from_numpy(y).pin_memory().numpy() for y in Yp]
        else:
            Yin = Yp
        out, secs = p.sweep_host(Yin)
        assert secs > 0
        for n in range(3):
            assert rel_fro(out[n], ref[n]) < 1e-6
    p.close()


def test_auto_layout_picks_ncopy_when_it_fits():
    """layout="auto" resolves to NCopy for a tensor whose N+1 slabs fit the
    device-memory budget, and then holds the same copies and Yhat as an
    explicit NCopy plan (copies bit-exact; Yhat up to the order of the FP32
    atomics at row-run boundaries)."""
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf((3000, 500, 200), draws=30000, s=1.1, seed=31)
    T, R = 4, 16
    a = _plan(dims, vals, idx, T, R, layout="auto")
    b = _plan(dims, vals, idx, T, R, layout="ncopy")
    assert a.info()["layout"] == "ncopy"
    assert b.info()["layout"] == "ncopy"
    assert _plan(dims, vals, idx, T, R, layout="pingpong").info()["layout"] == "pingpong"
    rng = np.random.default_rng(5)
    for n in range(3):
        y = rng.uniform(-1, 1, (int(dims[n]), a.Rp)).astype(np.float32)
        a.set_factor(n, y)
        b.set_factor(n, y)
    for n in range(3):
        av, aix = a.copy(n)
        bv, bix = b.copy(n)
        assert np.array_equal(av, bv) and all(np.array_equal(x, y) for x, y in zip(aix, bix))
    a.sweep()
    b.sweep()
    for n in range(3):
        assert rel_fro(a.yhat(n), b.yhat(n)) < 1e-6, n
    a.close()
    b.close()
