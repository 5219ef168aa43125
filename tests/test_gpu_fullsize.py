"""The bench workload at its full size (Zipf(1.1) 1,000,000 x 200,000 x
50,000 from 100M draws, ~64.7M nonzeros, rank 32, 16 plan workers), checked
through properties that do not need an oracle run of the whole tensor:

* every remapped slab is a permutation of the input nonzeros (order-free
  checksums of values, indices and whole coordinates);
* the slab the next mode reads is grouped by that mode's shard, ascending;
* MTTKRP is linear in each gathered factor (scaling a factor by 2 is exact in
  FP32; the second sweep reads the slab in its next order, so sums differ
  only by FP32 summation order);
* sampled output rows agree with an FP64 sum over their nonzeros;
* the NCopy plan's copies hold the same nonzeros and give the same Yhat."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_fro

pytestmark = pytest.mark.gpu

DIMS = (1_000_000, 200_000, 50_000)
R = 32


def _workload():
    import torch
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf_torch(DIMS, 100_000_000, 1.1, 2, device="cuda")
    to = lambda t: t.cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)
    return np.asarray(to(dims), np.uint32), to(vals).astype(np.float32), \
        [to(i).astype(np.uint32) for i in idx]


def _checksums(vals, idx):
    """Order-free integer checksums of the nonzeros: value bit patterns,
    index columns, and a mix of whole coordinates with their values."""
    vb = np.asarray(vals, np.float32).view(np.uint32).astype(np.uint64)
    cols = [np.asarray(i, np.uint64) for i in idx]
    coord = (cols[0] * np.uint64(0x9E3779B97F4A7C15) + cols[1] * np.uint64(0xC2B2AE3D27D4EB4F)
             + cols[2] * np.uint64(0x165667B19E3779F9))
    mix = coord ^ (vb << np.uint64(17))
    return (int(vb.sum()), [int(c.sum()) for c in cols], int(np.bitwise_xor.reduce(mix)),
            int(mix.sum()), int((mix * mix).sum()))


def _factors(dims, Rp, seed=5):
    rng = np.random.default_rng(seed)
    Y = []
    for n, d in enumerate(dims):
        y = np.zeros((int(d), Rp), np.float32)
        y[:, :R] = rng.uniform(-1, 1, (int(d), R)).astype(np.float32)
        Y.append(y)
    return Y


def test_full_size_sweep_properties():
    import dynasor_plus_b200 as d
    dims, vals, idx = _workload()
    nnz = len(vals)
    assert nnz > 60_000_000
    ref = _checksums(vals, idx)
    p = d.Plan(dims, vals, idx, threads=16, rank=R, layout="pingpong")
    info = p.info()
    shift = info["mn_shift"]
    Y = _factors(dims, p.Rp)
    for n in range(3):
        p.set_factor(n, Y[n])
    yh = []
    for n in range(3):
        p.process(n)
        yh.append(p.yhat(n))
        sv, six = p.slab()
        assert _checksums(sv, six) == ref, n
        nm = (n + 1) % 3
        sh = six[nm] >> np.uint32(shift[nm])
        assert np.all(sh[1:] >= sh[:-1]), f"slab after mode {n} not grouped by mode-{nm} shard"
        del sv, six, sh
    # sampled rows of every mode against an FP64 sum over their nonzeros
    rng = np.random.default_rng(1)
    for n in range(3):
        rows = rng.choice(int(dims[n]), 64, replace=False)
        sel = np.isin(idx[n], rows)
        prod = vals[sel].astype(np.float64)[:, None] * np.ones((1, R))
        for w in range(3):
            if w != n:
                prod *= Y[w][idx[w][sel], :R].astype(np.float64)
        want = np.zeros((int(dims[n]), R))
        np.add.at(want, idx[n][sel], prod)
        got = yh[n][rows, :R].astype(np.float64)
        assert rel_fro(got, want[rows]) <= 1e-5, n
    # linearity: Y1 doubled doubles Yhat of modes 0 and 2, leaves mode 1
    Y2 = [y.copy() for y in Y]
    Y2[1] *= 2.0
    for n in range(3):
        p.set_factor(n, Y2[n])
    p.sweep()
    for n in range(3):
        scale = 1.0 if n == 1 else 2.0
        assert rel_fro(p.yhat(n), scale * yh[n]) <= 1e-5, n
    p.close()
    # NCopy: same nonzeros in every copy, same Yhat
    q = d.Plan(dims, vals, idx, threads=16, rank=R, layout="ncopy")
    for n in range(3):
        q.set_factor(n, Y[n])
        cv, cix = q.copy(n)
        assert _checksums(cv, cix) == ref, n
        sh = cix[n] >> np.uint32(shift[n])
        assert np.all(sh[1:] >= sh[:-1]), n
        del cv, cix, sh
    q.sweep()
    for n in range(3):
        assert rel_fro(q.yhat(n), yh[n]) <= 1e-5, n
    q.close()
