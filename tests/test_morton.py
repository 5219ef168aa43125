"""The Morton layout (build_morton_layout / spmttkrp_all_modes_morton,
src/dynasor_morton.cpp).

CPU: the oracle's bit plan, keys and key order equal the reference's
(build_morton_layout run here), so the oracle is pinned.
GPU: the device build gives the same masks, keys and values bit for bit;
the all-modes pass over the keys matches the FP64 oracle and the
reference's Morton driver; sweeps, downloads, CP-ALS (run as Jacobi, as the
reference does) and .dnp files of the layout."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_fro

TOL_FP32 = 1e-5


def _zipf(dims=(3000, 500, 200), draws=30000, seed=31):
    from dynasor_plus_b200 import synth
    return synth.zipf(dims, draws=draws, s=1.1, seed=seed)


def _distinct(dims, nnz, seed):
    """Up to nnz distinct uniform coordinates (any mode count), random order."""
    rng = np.random.default_rng(seed)
    coords = np.stack([rng.integers(0, int(d), size=int(nnz * 1.3), dtype=np.int64)
                       for d in dims], 1)
    _, first = np.unique(coords, axis=0, return_index=True)
    coords = coords[np.sort(first)[:nnz]]
    idx = [np.ascontiguousarray(coords[:, n], dtype=np.uint32) for n in range(len(dims))]
    vals = rng.standard_normal(len(coords)).astype(np.float32)
    return np.asarray(dims, np.uint32), vals, idx


CASES = [
    ("zipf3", lambda: _zipf()),
    ("mode4", lambda: _distinct((50, 700, 9, 3000), 40000, 3)),
    ("tiny-modes", lambda: _distinct((1, 2, 3, 5, 1000), 2000, 4)),
    ("mode2-wide", lambda: _distinct((1 << 20, 70000), 50000, 5)),
    # 22 + 21 + 21 = 64 key bits: the high word is fully used
    ("bits64", lambda: _distinct((1 << 22, 1 << 21, (1 << 21) - 5), 30000, 6)),
]


@pytest.mark.parametrize("name,make", CASES)
def test_oracle_morton_is_the_reference_layout(refb, name, make):
    dims, vals, idx = make()
    mine = refb.morton(dims, vals, idx)
    ref = refb.Reference(dims, vals, idx)
    ref.build(2, "pingpong")
    ref.build_morton()
    rm, rb, rk, rv = ref.morton()
    m, b, k, v = mine
    assert np.array_equal(m, rm) and np.array_equal(b, rb)
    assert np.array_equal(k, rk) and np.array_equal(v, rv)
    assert np.all(k[1:] >= k[:-1])


def test_oracle_rejects_more_than_64_key_bits(bindings):
    dims = np.array([1 << 22, 1 << 22, 1 << 22], np.uint32)     # 66 bits
    idx = [np.zeros(4, np.uint32) for _ in range(3)]
    assert bindings.morton(dims, np.ones(4, np.float32), idx) is None


@pytest.mark.gpu
@pytest.mark.parametrize("name,make", CASES)
def test_device_morton_build_matches_oracle(bindings, name, make):
    import dynasor_plus_b200 as d
    dims, vals, idx = make()
    p = d.Plan(dims, vals, idx, threads=4, rank=16, layout="morton")
    assert p.info()["layout"] == "morton"
    m, b, k, v = p.morton()
    om, ob, ok, ov = bindings.morton(dims, vals, idx)
    assert np.array_equal(m, om) and np.array_equal(b, ob)
    assert np.array_equal(k, ok) and np.array_equal(v, ov)
    # the slab view decodes the keys
    sv, six = p.slab()
    assert np.array_equal(sv, ov)
    order = np.lexsort(tuple(reversed(idx)))
    got = np.lexsort(tuple(reversed(six)))
    assert all(np.array_equal(a[order], c[got]) for a, c in zip(idx, six))
    p.close()


@pytest.mark.gpu
def test_device_morton_rejects_more_than_64_key_bits():
    import dynasor_plus_b200 as d
    dims = np.array([1 << 22, 1 << 22, 1 << 22], np.uint32)
    idx = [np.array([0, 1, 2], np.uint32) for _ in range(3)]
    with pytest.raises(d.DgpuError) as e:
        d.Plan(dims, np.ones(3, np.float32), idx, threads=2, rank=16, layout="morton")
    assert "64 key bits" in str(e.value)


@pytest.mark.gpu
def test_morton_single_nonzero_and_two_modes():
    import dynasor_plus_b200 as d
    dims = np.array([7, 5], np.uint32)
    idx = [np.array([6], np.uint32), np.array([4], np.uint32)]
    vals = np.array([2.5], np.float32)
    p = d.Plan(dims, vals, idx, threads=1, rank=16, layout="morton")
    m, b, k, v = p.morton()
    assert list(b) == [3, 3] and v[0] == np.float32(2.5)
    Y = [np.zeros((int(n), 16), np.float32) for n in dims]
    Y[0][6, :] = 2.0
    Y[1][4, :] = 3.0
    for n in range(2):
        p.set_factor(n, Y[n])
    p.all_modes()
    assert np.allclose(p.yhat(0)[6], 2.5 * 3.0) and np.allclose(p.yhat(1)[4], 2.5 * 2.0)
    assert np.count_nonzero(p.yhat(0)) == 16 and np.count_nonzero(p.yhat(1)) == 16
    p.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,make", CASES[:3])
def test_all_modes_on_morton_matches_fp64_and_reference(refb, name, make):
    import dynasor_plus_b200 as d
    dims, vals, idx = make()
    R = 16
    p = d.Plan(dims, vals, idx, threads=4, rank=R, layout="morton")
    Y = refb.uniform_factors(5, dims, R)
    for n in range(len(dims)):
        p.set_factor(n, Y[n])
    p.all_modes()
    ref = refb.Reference(dims, vals, idx)
    ref.build(4, "pingpong")
    ref.build_morton()
    ref.factors(R)
    for n in range(len(dims)):
        ref.set_Y(n, Y[n])
    ref.all_modes_morton()
    for n in range(len(dims)):
        want = refb.mttkrp_f64(vals, idx, n, Y, R, int(dims[n]))
        got = p.yhat(n)
        assert rel_fro(got[:, :R], want[:, :R]) <= TOL_FP32, n
        assert rel_fro(got[:, :R], ref.yhat(n)[:, :R]) <= TOL_FP32, n
    # a sweep on Morton is the all-modes pass (equal up to the order of the
    # FP32 atomics); single modes are refused
    before = [p.yhat(n) for n in range(len(dims))]
    p.sweep()
    for n in range(len(dims)):
        assert rel_fro(p.yhat(n), before[n]) <= TOL_FP32
    with pytest.raises(d.DgpuError):
        p.process(0)
    p.close()


@pytest.mark.gpu
def test_cpals_on_morton_runs_jacobi():
    """Gauss-Seidel requested on a Morton plan runs Jacobi (the reference's
    rule); the trajectory is the Jacobi one of a PingPong plan."""
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.cp_truth((300, 200, 100), 60_000, 4, 0.01, seed=3)
    R = 8
    m = d.Plan(dims, vals, idx, threads=4, rank=R, layout="morton")
    pp = d.Plan(dims, vals, idx, threads=4, rank=R, layout="pingpong")
    a = m.cpals(max_iters=3, tol=0.0, seed=42, kernel="gs")
    b = pp.cpals(max_iters=3, tol=0.0, seed=42, kernel="jacobi")
    assert len(a["fit_history"]) == len(b["fit_history"]) == 3
    assert np.max(np.abs(a["fit_history"] - b["fit_history"])) < 1e-5
    for n in range(3):
        assert rel_fro(m.factor(n), pp.factor(n)) < 1e-4
    m.close()
    pp.close()


@pytest.mark.gpu
def test_morton_dnp_round_trip_and_reference_bytes(refb, tmp_path):
    import dynasor_plus_b200 as d
    dims, vals, idx = _zipf(seed=9)
    T, R = 4, 16
    ref = refb.Reference(dims, vals, idx)
    ref.build(T, "pingpong")
    ref.build_morton()
    rpath = tmp_path / "ref_morton.dnp"
    assert ref.save_dnp(rpath)
    assert d.dnp_peek(rpath)["layout"] == "morton"
    p = d.Plan(dims, vals, idx, threads=T, rank=R, layout="morton")
    mine = tmp_path / "mine.dnp"
    p.save_dnp(mine)
    assert mine.read_bytes() == rpath.read_bytes()
    q = d.Plan.from_dnp(rpath, threads=T, rank=R)
    assert q.info()["layout"] == "morton"
    for x, y in zip(p.morton(), q.morton()):
        assert np.array_equal(x, y)
    Y = refb.uniform_factors(2, dims, R)
    for n in range(3):
        p.set_factor(n, Y[n])
        q.set_factor(n, Y[n])
    p.all_modes()
    q.all_modes()
    for n in range(3):
        assert rel_fro(q.yhat(n), p.yhat(n)) <= TOL_FP32
    # the reference reads this engine's file
    r2 = refb.Reference.from_dnp(mine, T)
    assert r2 is not None
    assert all(np.array_equal(x, y) for x, y in zip(r2.morton(), ref.morton()))
    p.close()
    q.close()
