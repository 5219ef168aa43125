"""CP-OPT forward (model at the nonzeros) and adjoint (MTTKRP minus
Y * Hadamard-of-Grams) through a torch.autograd.Function that lives in the
test harness only.  Checked against FP64 central finite differences and
against a gradient assembled from the reference's own MTTKRP."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _loss64(bindings, idx, vals, Y, R):
    """0.5 * ||X - M||_F^2 over all cells, FP64, from FP32 factors."""
    x = vals.astype(np.float64)
    m = bindings.model_values(idx, Y, R)
    G = [y[:, :R].astype(np.float64).T @ y[:, :R].astype(np.float64) for y in Y]
    H = np.ones((R, R))
    for Gn in G:
        H *= Gn
    return 0.5 * (x @ x) - x @ m + 0.5 * H.sum()


def _make(seed=3, dims=(60, 50, 40), nnz=4000, R=8):
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform(dims, nnz, seed=seed, values="normal")
    rng = np.random.default_rng(seed)
    Rp = (R + 15) // 16 * 16
    Y = []
    for d in dims:
        y = np.zeros((int(d), Rp), np.float32)
        y[:, :R] = rng.normal(0, 0.1, (int(d), R))
        Y.append(y)
    return dims, vals, idx, Y, R


class CpOptLoss:
    """torch.autograd.Function: forward evaluates the CP model at the
    nonzeros on the GPU (dgpu_model_values); backward returns the
    dgpu_cpopt_gradient factors.  Test harness only."""

    @staticmethod
    def build(plan, vals, R):
        import torch

        class _F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, *Ys):
                for n, y in enumerate(Ys):
                    plan.set_factor(n, y.detach().cpu().numpy())
                m = plan.model_values().astype(np.float64)
                slab_v, _ = plan.slab()
                x = slab_v.astype(np.float64)
                G = [y.detach().double()[:, :R].T @ y.detach().double()[:, :R] for y in Ys]
                H = torch.ones(R, R, dtype=torch.float64)
                for Gn in G:
                    H = H * Gn
                loss = 0.5 * float(x @ x) - float(x @ m) + 0.5 * float(H.sum())
                return torch.tensor(loss, dtype=torch.float64)

            @staticmethod
            def backward(ctx, gout):
                grads = plan.cpopt_gradient()
                return tuple(torch.from_numpy(g).double() * gout for g in grads)

        return _F


def test_gradient_vs_finite_differences(bindings):
    import torch
    import dynasor_plus_b200 as d
    dims, vals, idx, Y, R = _make()
    p = d.Plan(dims, vals, idx, threads=4, rank=R)
    F = CpOptLoss.build(p, vals, R)
    Ys = [torch.tensor(y, requires_grad=True) for y in Y]
    loss = F.apply(*Ys)
    lv = float(loss.detach())
    assert abs(lv - _loss64(bindings, idx, vals, Y, R)) < 1e-3 * max(1.0, abs(lv))
    loss.backward()
    rng = np.random.default_rng(0)
    h = 1e-4
    worst = 0.0
    for _ in range(64):
        n = int(rng.integers(0, 3))
        i = int(rng.integers(0, int(dims[n])))
        r = int(rng.integers(0, R))
        # central difference in FP64 on FP64 copies of the factors
        Yp = [y.astype(np.float64) for y in Y]
        Ym = [y.astype(np.float64) for y in Y]
        Yp[n][i, r] += h
        Ym[n][i, r] -= h
        fd = (_loss64_f64(bindings, idx, vals, Yp, R) - _loss64_f64(bindings, idx, vals, Ym, R)) / (2 * h)
        g = float(Ys[n].grad[i, r])
        worst = max(worst, abs(g - fd) / max(1.0, abs(fd)))
    assert worst < 1e-3, worst


def _loss64_f64(bindings, idx, vals, Y, R):
    x = vals.astype(np.float64)
    N = len(Y)
    m = np.zeros(len(x))
    prod = np.ones((len(x), R))
    for n in range(N):
        prod *= Y[n][idx[n], :R]
    m = prod.sum(1)
    H = np.ones((R, R))
    for y in Y:
        H *= y[:, :R].T @ y[:, :R]
    return 0.5 * (x @ x) - x @ m + 0.5 * H.sum()


def test_gradient_vs_reference_mttkrp(refb):
    import dynasor_plus_b200 as d
    dims, vals, idx, Y, R = _make(seed=5)
    p = d.Plan(dims, vals, idx, threads=4, rank=R)
    for n in range(3):
        p.set_factor(n, Y[n])
    g = p.cpopt_gradient()
    ref = refb.Reference(dims, vals, idx)
    ref.build(4, "pingpong")
    ref.factors(R)
    for n in range(3):
        ref.set_Y(n, Y[n])
    ref.reference_mttkrp()
    for n in range(3):
        H = np.ones((R, R))
        for m in range(3):
            if m != n:
                H *= Y[m][:, :R].astype(np.float64).T @ Y[m][:, :R]
        expect = Y[n][:, :R].astype(np.float64) @ H - ref.yhat(n)[:, :R]
        err = np.linalg.norm(g[n][:, :R] - expect) / np.linalg.norm(expect)
        assert err < 1e-5, (n, err)


def test_model_values_vs_oracle(bindings):
    import dynasor_plus_b200 as d
    dims, vals, idx, Y, R = _make(seed=9)
    p = d.Plan(dims, vals, idx, threads=2, rank=R)
    for n in range(3):
        p.set_factor(n, Y[n])
    m = p.model_values()
    v, ix = p.slab()
    m64 = bindings.model_values(ix, Y, R)
    assert np.max(np.abs(m - m64)) < 1e-5 * max(1.0, np.max(np.abs(m64)))


def test_outputs_into_caller_buffers_match_fresh_ones():
    """model_values / cpopt_gradient written into the caller's arrays (the
    copies go through the plan's pinned chunks, here across several 8 MB
    chunks) equal freshly allocated results, on two calls in a row; a
    buffer of the wrong shape or type is refused."""
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((60000, 50000, 400), 3_000_000, seed=5, values="normal")
    rng = np.random.default_rng(6)
    R = 32
    # NCopy: the slab order (and so the order of the model values) stays
    # put across the gradient's mode passes
    p = d.Plan(dims, vals, idx, threads=4, rank=R, layout="ncopy")
    for n in range(3):
        y = np.zeros((int(dims[n]), p.Rp), np.float32)
        y[:, :R] = rng.normal(0, 0.1, (int(dims[n]), R))
        p.set_factor(n, y)
    m0 = p.model_values()
    g0 = p.cpopt_gradient()
    mo = np.full(p.nnz, np.nan, np.float32)
    go = [np.full_like(g, np.nan) for g in g0]
    for _ in range(2):
        assert p.model_values(out=mo) is mo
        assert np.array_equal(mo, m0)
        assert p.cpopt_gradient(out=go) is go
        for a, b in zip(go, g0):
            assert np.allclose(a, b, rtol=1e-5, atol=1e-6)
    with pytest.raises(ValueError):
        p.model_values(out=np.zeros(p.nnz - 1, np.float32))
    with pytest.raises(ValueError):
        p.cpopt_gradient(out=[g.astype(np.float64) for g in g0])
    p.close()
