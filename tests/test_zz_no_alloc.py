"""dgpu_sort_slab_noalloc: the stable shard partition for callers that may
not allocate device memory (their device memory belongs to a host
framework's pool, or cudaMalloc's device-wide synchronisation is not
allowed on their path).  It must give exactly the slab that the plan API
builds with its own (allocating) partition: the initial mode-0 shard order
of dgpu_plan_create.  Integer work, so bit-exact, on two calls in a row
(the second reuses the fixed scratch left by the first).

Kept in a file that pytest collects last."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sort_noalloc(vals, idx, key_mode, key_shift, nb):
    import torch
    import dynasor_plus_b200 as d
    N = len(idx)
    vin = torch.from_numpy(np.ascontiguousarray(vals, np.float32)).cuda()
    iin = [torch.from_numpy(np.ascontiguousarray(i, np.uint32).view(np.int32)).cuda() for i in idx]
    vout = torch.full_like(vin, float("nan"))
    iout = [torch.full_like(x, -1) for x in iin]
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    pin = (C.c_void_p * N)(*[x.data_ptr() for x in iin])
    pout = (C.c_void_p * N)(*[x.data_ptr() for x in iout])
    d.check(d.lib().dgpu_sort_slab_noalloc(C.c_void_p(stream.cuda_stream), N, len(vals),
                                           C.c_void_p(vin.data_ptr()), pin,
                                           C.c_void_p(vout.data_ptr()), pout,
                                           key_mode, key_shift, nb))
    torch.cuda.synchronize()
    return vout.cpu().numpy(), [x.cpu().numpy().view(np.uint32) for x in iout]


def test_noalloc_partition_matches_plan_build_twice():
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    for call, (dims, nnz, T) in enumerate([((5000, 300, 200), 40000, 4),
                                           ((900, 700, 60, 40), 25000, 16)]):
        dims, vals, idx = synth.uniform(dims, nnz, seed=70 + call)
        plan = d.Plan(dims, vals, idx, threads=T, rank=8)
        inf = plan.info()
        ref_v, ref_i = plan.slab()           # the plan API's own stable mode-0 partition
        plan.close()
        v, ix = _sort_noalloc(vals, idx, 0, inf["mn_shift"][0], inf["shards_per_mode"][0])
        assert np.array_equal(v, ref_v), call
        for n in range(len(dims)):
            assert np.array_equal(ix[n], ref_i[n]), (call, n)


def test_noalloc_multi_block_scan_matches_stable_argsort():
    """~1M nonzeros in 2048 buckets: 245 tiles x 2048 buckets = 501,760
    counters, 31 blocks of the counter scan (the block sums are scanned and
    added back), against numpy's stable argsort by key, twice in a row."""
    from dynasor_plus_b200 import synth
    shift = 3
    dims, vals, idx = synth.uniform((2048 << shift, 300, 200), 1_000_000, seed=81)
    key = idx[0] >> shift
    order = np.argsort(key, kind="stable")
    for _ in range(2):
        v, ix = _sort_noalloc(vals, idx, 0, shift, 2048)
        assert np.array_equal(v, vals[order])
        for n in range(3):
            assert np.array_equal(ix[n], idx[n][order]), n


def test_noalloc_rejects_oversized_and_bad_keys():
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((100, 50, 20), 2000, seed=1)
    with pytest.raises(d.DgpuError) as e:          # keys up to 99 >= 64 buckets
        _sort_noalloc(vals, idx, 0, 0, 64)
    assert e.value.code == -5
    with pytest.raises(d.DgpuError) as e:          # more buckets than one pass handles
        _sort_noalloc(vals, idx, 0, 0, 4096)
    assert e.value.code == -1
    big = 5_000_000                                # 2048 x 1221 tiles > the fixed scratch
    dims, vals, idx = synth.uniform((4096, 10, 10), big, seed=2)
    with pytest.raises(d.DgpuError) as e:
        _sort_noalloc(vals, idx, 0, 1, 2048)
    assert e.value.code == -1 and "scratch" in str(e.value)


def test_noalloc_rejects_a_capturing_stream():
    """The call ends with a blocking read of its fault flag, which a stream
    capture cannot hold: on a capturing stream it queues nothing and gives
    DGPU_ERR_ARG."""
    import torch
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((64, 50, 20), 3000, seed=3)
    vin = torch.from_numpy(vals).cuda()
    iin = [torch.from_numpy(i.view(np.int32)).cuda() for i in idx]
    vout = torch.empty_like(vin)
    iout = [torch.empty_like(x) for x in iin]
    pin = (C.c_void_p * 3)(*[x.data_ptr() for x in iin])
    pout = (C.c_void_p * 3)(*[x.data_ptr() for x in iout])
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        rc = d.lib().dgpu_sort_slab_noalloc(C.c_void_p(s.cuda_stream), 3, len(vals),
                                            C.c_void_p(vin.data_ptr()), pin,
                                            C.c_void_p(vout.data_ptr()), pout, 0, 0, 64)
        vout.add_(0.0)                      # keep the captured graph non-empty
    assert rc == -1
    assert b"captured" in d.lib().dgpu_last_error()
