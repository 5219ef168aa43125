"""Processed-tensor files (.dnp, the reference's runtime-only mode,
src/dynasor_dnp.cpp).

CPU: the header reader and every rejection that happens before the device
is touched, on files the reference itself writes (save_dnp_tensor).
GPU: a plan saved by this engine is byte-identical to the reference's file
for the same tensor, threads and layout; a plan loaded from the reference's
file sweeps to the same slabs and Yhat as one built from the COO; the
reference loads this engine's files."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_fro

ERR_ARG, ERR_IO = -1, -7


def _tensor(seed=31, dims=(3000, 500, 200), draws=30000):
    from dynasor_plus_b200 import synth
    return synth.zipf(dims, draws=draws, s=1.1, seed=seed)


def _ref_file(refb, tmp_path, layout, threads=4, seed=31, name=None):
    dims, vals, idx = _tensor(seed)
    ref = refb.Reference(dims, vals, idx)
    ref.build(threads, layout)
    path = tmp_path / (name or f"ref_{layout}_{threads}.dnp")
    assert ref.save_dnp(path)
    return path, (dims, vals, idx), ref


@pytest.mark.parametrize("layout", ["pingpong", "ncopy"])
def test_peek_reads_the_reference_header(refb, tmp_path, layout):
    import dynasor_plus_b200 as d
    path, (dims, vals, _), _ = _ref_file(refb, tmp_path, layout, threads=6)
    info = d.dnp_peek(path)
    assert info == {"layout": layout, "num_modes": 3, "nnz": len(vals),
                    "mode_size": [int(x) for x in dims], "num_threads": 6}


def test_rejections_before_the_device(refb, tmp_path):
    import dynasor_plus_b200 as d
    path, _, _ = _ref_file(refb, tmp_path, "pingpong", threads=4)
    # the schedule is thread-specific: another thread count is refused
    with pytest.raises(d.DgpuError) as e:
        d.Plan.from_dnp(path, threads=8, rank=16)
    assert e.value.code == ERR_ARG and "4 threads" in str(e.value)
    # InPlace files are not a layout this engine runs
    ip, _, _ = _ref_file(refb, tmp_path, "inplace", threads=4)
    assert d.dnp_peek(ip)["layout"] == "inplace"
    with pytest.raises(d.DgpuError) as e:
        d.Plan.from_dnp(ip, threads=4, rank=16)
    assert e.value.code == ERR_ARG and "InPlace" in str(e.value)
    # bad magic, truncated body, missing file
    raw = path.read_bytes()
    bad = tmp_path / "bad.dnp"
    bad.write_bytes(b"XNP1" + raw[4:])
    with pytest.raises(d.DgpuError) as e:
        d.dnp_peek(bad)
    assert e.value.code == ERR_IO
    cut = tmp_path / "cut.dnp"
    cut.write_bytes(raw[: len(raw) - 1000])
    assert d.dnp_peek(cut)["nnz"] > 0          # the header is intact
    with pytest.raises(d.DgpuError) as e:
        d.Plan.from_dnp(cut, threads=4, rank=16)
    assert e.value.code == ERR_IO and "truncated" in str(e.value)
    with pytest.raises(d.DgpuError) as e:
        d.dnp_peek(tmp_path / "missing.dnp")
    assert e.value.code == ERR_IO
    # a header whose shard geometry does not fit its mode size
    geo = bytearray(raw)
    hdr = 4 + 5 * 4 + 8 + 8 * 4 + 4 + 8 + 14 * 4        # fixed header bytes
    geo[hdr:hdr + 4] = (7).to_bytes(4, "little")       # shards of mode 0
    bg = tmp_path / "geo.dnp"
    bg.write_bytes(bytes(geo))
    with pytest.raises(d.DgpuError) as e:
        d.Plan.from_dnp(bg, threads=4, rank=16)
    assert e.value.code == ERR_IO and "geometry" in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["pingpong", "ncopy"])
@pytest.mark.parametrize("threads", [1, 4])
def test_saved_file_is_the_reference_file(refb, tmp_path, layout, threads):
    """Same tensor, threads and layout: this engine writes the reference's
    bytes (shard tables, schedule, cursor table, touched bitmaps, slab(s),
    NCopy row pointers)."""
    import dynasor_plus_b200 as d
    path, (dims, vals, idx), _ = _ref_file(refb, tmp_path, layout, threads=threads)
    p = d.Plan(dims, vals, idx, threads=threads, rank=16, layout=layout)
    mine = tmp_path / "mine.dnp"
    p.save_dnp(mine)
    a, b = mine.read_bytes(), path.read_bytes()
    assert len(a) == len(b)
    if a != b:
        first = next(i for i in range(len(a)) if a[i] != b[i])
        pytest.fail(f"files differ first at byte {first} of {len(a)}")
    p.close()


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["pingpong", "ncopy"])
def test_plan_from_reference_file_sweeps_like_a_built_plan(refb, tmp_path, layout):
    import dynasor_plus_b200 as d
    T, R = 4, 16
    path, (dims, vals, idx), ref = _ref_file(refb, tmp_path, layout, threads=T)
    a = d.Plan.from_dnp(path, threads=T, rank=R)
    b = d.Plan(dims, vals, idx, threads=T, rank=R, layout=layout)
    ia, ib = a.info(), b.info()
    for k in ("num_modes", "nnz", "mode_size", "mn_shift", "shards_per_mode", "kernel_class",
              "layout"):
        assert ia[k] == ib[k], k
    for n in range(3):
        assert all(np.array_equal(x, y) for x, y in zip(a.shards(n), b.shards(n)))
    rng = np.random.default_rng(2)
    Y = [rng.uniform(-1, 1, (int(dims[n]), a.Rp)).astype(np.float32) for n in range(3)]
    Yr = refb.uniform_factors(9, dims, R)
    ref.factors(R)
    for n in range(3):
        a.set_factor(n, Y[n])
        b.set_factor(n, Y[n])
    for sweep in range(2):
        for n in range(3):
            a.process(n)
            b.process(n)
            assert rel_fro(a.yhat(n), b.yhat(n)) < 1e-6, (sweep, n)
            if layout == "pingpong":
                va, ixa = a.slab()
                vb, ixb = b.slab()
                assert np.array_equal(va, vb) and all(np.array_equal(x, y) for x, y in zip(ixa, ixb))
    # and against the reference's own sweep on the loaded tensor
    r2 = refb.Reference.from_dnp(path, T)
    assert r2 is not None
    r2.factors(R)
    c = d.Plan.from_dnp(path, threads=T, rank=R)
    for n in range(3):
        r2.set_Y(n, Yr[n])
        c.set_factor(n, Yr[n])
    r2.sweep_begin()
    for n in range(3):
        r2.process(n)
        c.process(n)
        assert rel_fro(c.yhat(n)[:, :R], r2.yhat(n)[:, :R]) <= 1e-5, n
    for p in (a, b, c):
        p.close()


@pytest.mark.gpu
def test_reference_loads_a_file_saved_after_sweeps(refb, tmp_path):
    """A PingPong plan saved after two sweeps (slab in a later mode-0 order)
    is a valid runtime file for the reference too: its sweep from the loaded
    state matches this engine's plan continuing from the same state."""
    import dynasor_plus_b200 as d
    T, R = 4, 16
    dims, vals, idx = _tensor(7)
    p = d.Plan(dims, vals, idx, threads=T, rank=R)
    Y = refb.uniform_factors(3, dims, R)
    for n in range(3):
        p.set_factor(n, Y[n])
    p.sweep()
    p.sweep()
    path = tmp_path / "after.dnp"
    p.save_dnp(path)
    r = refb.Reference.from_dnp(path, T)
    assert r is not None
    r.factors(R)
    for n in range(3):
        r.set_Y(n, Y[n])
    r.sweep_begin()
    for n in range(3):
        r.process(n)
        p.process(n)
        assert rel_fro(p.yhat(n)[:, :R], r.yhat(n)[:, :R]) <= 1e-5, n
        v, ix = p.slab()
        rv, rix = r.slab()
        assert np.array_equal(v, rv) and all(np.array_equal(x, y) for x, y in zip(ix, rix)), n
    # a PingPong plan in the middle of a sweep is not saved
    p.process(0)
    with pytest.raises(d.DgpuError):
        p.save_dnp(tmp_path / "mid.dnp")
    p.close()
