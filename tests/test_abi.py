"""The C-ABI library loads on a machine without a GPU, exports every symbol
declared in include/*.h, fails loudly (no CPU fallback) when no device is
present, and its host-only loaders follow the reference's formats."""
from __future__ import annotations

import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT, HAS_GPU, load_golden


def _declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(dgpu_[a-z0-9_]+)\s*\(", txt):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol():
    import dynasor_plus_b200 as d
    L = C.CDLL(d.LIB_PATH)
    syms = _declared_symbols()
    assert len(syms) > 30
    missing = [s for s in sorted(syms) if not hasattr(L, s)]
    assert not missing, missing


def test_python_binding_covers_declared_symbols():
    from dynasor_plus_b200 import _lib
    assert _declared_symbols() <= set(_lib._SIGS)


def test_version_and_error_string():
    from dynasor_plus_b200 import _lib
    L = _lib.lib()
    assert L.dgpu_version() >= 0x000100
    assert L.dgpu_plan_create(None, None, None) == -1
    assert b"null" in L.dgpu_last_error()


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_no_device_fails_loudly():
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((10, 10, 10), 50, seed=1)
    with pytest.raises(d.DgpuError) as e:
        d.Plan(dims, vals, idx, threads=2, rank=8)
    assert e.value.code == -2


def test_tns_loader_and_dnb_roundtrip(tmp_path):
    import dynasor_plus_b200 as d
    g = load_golden("ref_3d7_T2_R16.npz")
    dims = g["dims"]
    path = tmp_path / "t.tns"
    with open(path, "w") as f:
        f.write("# comment line\n\n")
        for k in range(len(g["vals"])):
            f.write(" ".join(str(int(g[f"idx{n}"][k]) + 1) for n in range(3)))
            f.write(f" {float(g['vals'][k]):.6f}\n")
    dd, vv, ii = d.load_coo_tensor(str(path), cache=True)
    assert np.array_equal(dd, dims)
    assert np.array_equal(vv, g["vals"])
    for n in range(3):
        assert np.array_equal(ii[n], g[f"idx{n}"])
    assert os.path.exists(str(path) + ".dnb")
    d2, v2, i2 = d.load_dnb(str(path) + ".dnb")
    assert np.array_equal(d2, dims) and np.array_equal(v2, vv)
    # the cached path is taken on the second load
    d3, v3, _ = d.load_coo_tensor(str(path), cache=True)
    assert np.array_equal(v3, vv)


def test_splatt_header_sets_mode_sizes(tmp_path):
    import dynasor_plus_b200 as d
    path = tmp_path / "h.tns"
    path.write_text("3\n10 20 30\n1 2 3 1.5\n4 5 6 -2\n")
    dims, vals, idx = d.load_coo_tensor(str(path), cache=False)
    assert list(dims) == [10, 20, 30]
    assert list(vals) == [1.5, -2.0]
    assert list(idx[2]) == [2, 5]


@pytest.mark.parametrize("text", ["1 2 x\n", "0 1 1 1.0\n", "1 1 1 1\n1 1 1\n"])
def test_malformed_tns_rejected(tmp_path, text):
    import dynasor_plus_b200 as d
    path = tmp_path / "bad.tns"
    path.write_text(text)
    with pytest.raises(d.DgpuError) as e:
        d.load_coo_tensor(str(path), cache=False)
    assert e.value.code in (-7, -4)


def test_truncated_dnb_rejected(tmp_path):
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((5, 6, 7), 100, seed=3)
    p = str(tmp_path / "x.dnb")
    d.save_dnb_tensor(p, dims, vals, idx)
    d2, v2, i2 = d.load_dnb(p)
    assert np.array_equal(v2, vals) and all(np.array_equal(a, b) for a, b in zip(i2, idx))
    raw = open(p, "rb").read()
    open(p, "wb").write(raw[: len(raw) - 10])
    with pytest.raises(d.DgpuError) as e:
        d.load_dnb(p)
    assert e.value.code == -7


def test_dnb_matches_reference_layout(tmp_path, refb):
    """A .dnb written here loads in the reference's own loader path
    (byte layout of src/dynasor_io.cpp:747-774)."""
    import struct
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((5, 6, 7), 30, seed=4)
    p = str(tmp_path / "y.dnb")
    d.save_dnb_tensor(p, dims, vals, idx)
    raw = open(p, "rb").read()
    assert raw[:4] == b"DNB1"
    ver, vb, ib, nm = struct.unpack("<4I", raw[4:20])
    nnz, = struct.unpack("<Q", raw[20:28])
    assert (ver, vb, ib, nm, nnz) == (1, 4, 4, 3, 30)
    hdr = 4 + 4 * 4 + 8 + 4 * 8 + 4 * 7
    assert len(raw) == hdr + 30 * 4 * 4


def test_factor_dump_strips_padding(tmp_path):
    import struct
    import dynasor_plus_b200 as d
    Y = np.arange(5 * 16, dtype=np.float32).reshape(5, 16)
    p = str(tmp_path / "f.bin")
    d.dump_factor_matrix_bin(p, Y, 3)
    raw = open(p, "rb").read()
    assert raw[:4] == b"DYFM"
    ver, vb, r = struct.unpack("<3I", raw[4:16])
    rows, = struct.unpack("<Q", raw[16:24])
    assert (ver, vb, r, rows) == (1, 4, 3, 5)
    data = np.frombuffer(raw[24:], np.float32).reshape(5, 3)
    assert np.array_equal(data, Y[:, :3])
