"""The compute plan (dyn_build_compute_plan, src/dynasor_preprocess.cpp:
1179-1399) on the CPU: every clause of the CP-ALS kernel rule, the
keyword and environment overrides, the per-mode kernel class, the banner,
and the same decisions as the compiled reference's own function on
tensors built by the reference."""
from __future__ import annotations

import numpy as np
import pytest

GiB = 1 << 30


def _decide(**kw):
    import dynasor_plus_b200 as d
    base = dict(dims=(2000, 1500, 1000), nnz=2_000_000, rank=16, threads=8, layout="pingpong",
                host_avail_bytes=64 * GiB)
    base.update(kw)
    return d.compute_plan_decide(**base)


def test_auto_rule_clauses(monkeypatch):
    monkeypatch.delenv("DYN_CP_KERNEL", raising=False)
    c = _decide(layout="morton")
    assert (c["kernel"], c["kernel_reason"]) == ("jacobi", "forced-jacobi-by-layout")
    c = _decide(nnz=999_999)
    assert (c["kernel"], c["kernel_reason"]) == ("gs", "nnz<1M (linalg-dominated)")
    c = _decide(rank=64)
    assert (c["kernel"], c["kernel_reason"]) == ("gs", "all-modes-fallback-shape")
    c = _decide(rank=48)
    assert c["kernel"] == "jacobi"                       # N = 3, Rp 48 < 64
    c = _decide(dims=(200, 200, 200, 200), rank=128)
    assert (c["kernel"], c["kernel_reason"]) == ("gs", "all-modes-fallback-shape")
    c = _decide(dims=(200, 200, 200, 200), rank=64)
    assert c["kernel"] == "jacobi"                       # N = 4, Rp 64 < 128
    # the reference's per-thread output copies against min(avail / 4, 8 GiB)
    dims = (1_000_000, 200_000, 50_000)
    c = _decide(dims=dims, rank=32, threads=16)
    assert c["ofibs_bytes"] == 16 * sum((I * 32 * 4 + 63) // 64 * 64 for I in dims)
    assert c["budget_bytes"] == 8 * GiB
    assert c["kernel"] == "jacobi"
    c = _decide(dims=dims, rank=32, threads=16, host_avail_bytes=8 * GiB)
    assert c["budget_bytes"] == 2 * GiB
    assert (c["kernel"], c["kernel_reason"]) == ("gs", "ofibs>budget")
    assert c["factor_bytes"] == sum(2 * I * 32 * 4 for I in dims)


def test_keywords_and_environment(monkeypatch):
    monkeypatch.delenv("DYN_CP_KERNEL", raising=False)
    for word in ("jacobi", "all-modes", "all_modes", "JS"):
        c = _decide(nnz=10, kernel=word)
        assert (c["kernel"], c["kernel_reason"], c["kernel_source"]) == \
            ("jacobi", "user-forced-jacobi", "cli-kernel")
    for word in ("gs", "gauss-seidel", "classical", "per-mode", "Per_Mode"):
        c = _decide(kernel=word)
        assert (c["kernel"], c["kernel_reason"]) == ("gs", "user-forced-gs")
    c = _decide(layout="morton", kernel="gs")
    assert (c["kernel"], c["kernel_reason"]) == ("jacobi", "user-wanted-gs-but-layout-forces-jacobi")
    c = _decide(kernel="no-such-kernel")
    assert (c["kernel"], c["kernel_source"]) == ("jacobi", "cli-kernel")
    c = _decide(kernel="auto")
    assert c["kernel_source"] == "auto"
    monkeypatch.setenv("DYN_CP_KERNEL", "gs")
    c = _decide(kernel="jacobi")
    assert (c["kernel"], c["kernel_source"]) == ("gs", "env-kernel")


def test_per_mode_class_and_banner(monkeypatch):
    import dynasor_plus_b200 as d
    monkeypatch.delenv("DYN_CP_KERNEL", raising=False)
    kc, afl = [2, 0, 1], [40.0, 3.0, 32.0]
    c = _decide(kernel_class=kc, avg_fiber_len=afl)
    assert c["per_mode"] == ["Fiber", "Element", "Fiber"]
    c = _decide(layout="ncopy", kernel_class=kc, avg_fiber_len=afl)
    assert c["per_mode"] == ["FiberCSR", "Element", "Fiber"]
    c = _decide(layout="ncopy", fiber=False, kernel_class=kc, avg_fiber_len=afl)
    assert c["per_mode"] == ["Fiber", "Element", "Fiber"]
    text = d.format_compute_plan(c, "[plan]")
    lines = text.strip().splitlines()
    assert all(l.startswith("[plan] ") for l in lines)
    assert any("kernel : GaussSeidel" in l or "kernel : Jacobi" in l for l in lines)
    assert "per-mode : [Fiber,Element,Fiber]" in text
    with pytest.raises(d.DgpuError):
        d.compute_plan_decide(dims=(10,) * 9, nnz=1, rank=4, threads=1)


@pytest.mark.parametrize("shape,nnz,rank,threads,layout", [
    ((300, 200, 100), 50_000, 16, 4, "pingpong"),         # nnz < 1M
    ((4000, 3000, 2000), 1_200_000, 16, 8, "pingpong"),   # all-modes fits
    ((4000, 3000, 2000), 1_200_000, 64, 8, "pingpong"),   # N = 3, Rp 64
    ((400, 300, 200, 50), 1_100_000, 32, 4, "ncopy"),     # 4 modes, NCopy copies
    ((60, 50, 40), 30_000, 16, 2, "ncopy"),
])
def test_same_decision_as_reference(refb, monkeypatch, shape, nnz, rank, threads, layout):
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    monkeypatch.delenv("DYN_CP_KERNEL", raising=False)
    dims, vals, idx = synth.uniform(shape, nnz, seed=31)
    ref = refb.Reference(dims, vals, idx)
    ref.build(threads, layout)
    Rp = refb.padded_rank(rank)
    for kernel in ("auto", "gs", "jacobi"):
        k_ref, reason_ref, per_ref = ref.compute_plan(Rp, layout, kernel)
        c = d.compute_plan_decide(dims, nnz, rank, threads, layout=layout,
                                  kernel_class=ref.kclass, avg_fiber_len=ref.afl, kernel=kernel)
        assert (1 if c["kernel"] == "jacobi" else 0) == k_ref, (kernel, c, reason_ref)
        assert c["kernel_reason"] == reason_ref
        assert [{"Element": 0, "Fiber": 1, "FiberCSR": 2}[x] for x in c["per_mode"]] == per_ref
