"""The benchmark configurations at their stated sizes, checked against the
FP64 oracle and the compiled reference (oracle/_ref):

* plain CP-ALS, 200 x 200 x 200, 100,000 distinct nonzeros from a rank-5
  U(0,1) model plus 1% noise, rank 16, 50 Gauss-Seidel iterations, tol 1e-4;
* the skewed MTTKRP tensor, 1,000,000 x 200,000 x 50,000 from 100M Zipf(1.1)
  draws (~64.7M nonzeros), rank 32, 16 workers: the slab after every
  process(n) of one sweep bit for bit against the reference's
  SpmttkrpSweep, Yhat against FP64 and the reference;
* the 4-mode mixed-precision tensor, 50,000 x 20,000 x 2,000 x 500 from
  200M draws, rank 64, BF16 gathers with FP64 solves: one Gauss-Seidel and
  one Jacobi iteration against the FP64 oracle, per factor and fit;
* the CP-OPT gradient on 100,000 x 100,000 x 1,000 with 20M nonzeros, rank
  32: 64 central differences in FP64 and the gradient built from the
  reference's spmttkrp_reference;
* 16 restarts of rank 16 on 400,000 x 300,000 x 2,000 (50M Zipf(1.0)
  draws): restarts against FP64 CP-ALS runs from the same seeds;
* 32 tensors of uneven size in one batch against single runs and FP64.

Each check prints the errors it measured (pytest -s shows them)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_fro

pytestmark = pytest.mark.gpu

FIT_TOL = 1e-4          # north-star fit bound against FP64


def _host(t):
    import torch
    return t.cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


# ---------------------------------------------------------------------------
#  plain CP-ALS, 200^3, 100k nonzeros, rank 16, 50 iterations, tol 1e-4
# ---------------------------------------------------------------------------
def _c1():
    from dynasor_plus_b200 import synth
    return synth.cp_truth((200, 200, 200), 100_000, 5, 0.01, seed=1)


def test_plain_cpals_matches_reference_and_fp64(refb):
    """Same seed-42 N(0,1) initialisation as the reference's cpals (its only
    initialisation): the GPU fit trajectory against the reference's printed
    fits and against FP64 CP-ALS, stop iteration included."""
    import dynasor_plus_b200 as d
    dims, vals, idx = _c1()
    R, iters, tol, T = 16, 50, 1e-4, 8
    p = d.Plan(dims, vals, idx, threads=T, rank=R)
    r = p.cpals(max_iters=iters, tol=tol, seed=42)
    ref = refb.Reference(dims, vals, idx)
    ref.build(T, "pingpong")
    fit_ref, _, _, _ = ref.cpals(R, iters, tol, 42)
    fit64, Y64, lam64 = refb.cpals_f64(dims, vals, idx, R, iters, tol, seed=42)
    h = r["fit_history"]
    print(f"\nplain CP-ALS: iters gpu {len(h)} ref {len(fit_ref)} fp64 {len(fit64)}; "
          f"max |fit - ref| {np.max(np.abs(h - fit_ref[:len(h)])):.2e}, "
          f"max |fit - fp64| {np.max(np.abs(h - fit64[:len(h)])):.2e}")
    assert len(h) == len(fit_ref) == len(fit64)
    assert np.max(np.abs(h - fit_ref)) < FIT_TOL
    assert np.max(np.abs(h - fit64)) < 1e-6
    for n in range(3):
        assert rel_fro(p.factor(n)[:, :R], Y64[n][:, :R]) < 1e-4
    assert rel_fro(r["lambda"][:R], lam64) < 1e-4
    p.close()


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_plain_cpals_uniform_init_against_fp64(bindings, precision):
    """The configuration's own initialisation, U(0,1) factors from a fixed
    seed (uploaded, use_init), 50 iterations with tol 1e-4.  FP32 gathers
    follow FP64 CP-ALS; BF16 gathers keep the fit within 1e-4 of FP64 at
    every iteration and follow the FP64 run whose MTTKRP reads BF16-rounded
    factors (the last mode's FP32 ones, as BF16-gather CP-ALS does).
    (Per-factor errors against plain FP64 are large here for any precision:
    a rank-16 fit of rank-5 data is not unique.)"""
    import dynasor_plus_b200 as d
    dims, vals, idx = _c1()
    R = 16
    Y0 = bindings.uniform_factors(7, dims, R)
    p = d.Plan(dims, vals, idx, threads=8, rank=R, precision=precision)
    for n in range(3):
        p.set_factor(n, Y0[n])
    r = p.cpals(max_iters=50, tol=1e-4, seed=0, use_init=True)
    h = r["fit_history"]
    fit64, Y64, _ = bindings.cpals_f64(dims, vals, idx, R, 50, 1e-4, Y0=Y0)
    k = min(len(h), len(fit64))
    err = float(np.max(np.abs(h[:k] - fit64[:k])))
    print(f"\nplain CP-ALS U(0,1) init, {precision}: iters {len(h)} / fp64 {len(fit64)}, "
          f"final fit {h[-1]:.8f} vs {fit64[-1]:.8f}, max |dfit| {err:.2e}")
    assert err < FIT_TOL
    assert abs(h[-1] - fit64[-1]) < FIT_TOL
    if precision == "fp32":
        assert len(h) == len(fit64)
        assert err < 1e-6
        for n in range(3):
            assert rel_fro(p.factor(n)[:, :R], Y64[n][:, :R]) < 1e-4
    else:
        fb, Yb, _ = bindings.cpals_f64(dims, vals, idx, R, 50, 1e-4, Y0=Y0, bf16_gathers=True,
                                       last_mode_fp32=True)
        kb = min(len(h), len(fb))
        errb = float(np.max(np.abs(h[:kb] - fb[:kb])))
        print(f"  vs FP64 with BF16-rounded gathers: max |dfit| {errb:.2e}")
        # over 13 iterations FP32-level differences flip BF16 roundings of a
        # few factor entries (a 2^-9 relative step each): measured 1.2e-6
        assert errb < 1e-5
    p.close()


# ---------------------------------------------------------------------------
#  the skewed MTTKRP tensor at full size against the reference's sweep
# ---------------------------------------------------------------------------
def test_skewed_full_size_sweep_matches_reference(refb):
    """Two PingPong sweeps of the 64.7M-nonzero tensor, 16 workers, fiber
    sort on (the reference's defaults): after every process(n) the slab the
    next mode reads equals the reference's, value for value and index for
    index (the second sweep's partition passes run on the offset tables
    kept from the first cycle); in the first sweep Yhat[n] is within
    relative Frobenius 1e-5 of an FP64 MTTKRP and within the reference's
    own distance from FP64 (its parallel FP32 sums are not more exact than
    that) of the reference's Yhat."""
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.zipf_torch((1_000_000, 200_000, 50_000), 100_000_000, 1.1, 2,
                                       device="cuda")
    dims = np.asarray(_host(dims), np.uint32)
    T, R = 16, 32
    rng = np.random.default_rng(5)
    Rp = 32
    Y = []
    for dn in dims:
        y = np.zeros((int(dn), Rp), np.float32)
        y[:, :R] = rng.random((int(dn), R), dtype=np.float32)
        Y.append(y)
    ref = refb.Reference(dims, vals, idx)
    ref.build(T, "pingpong")
    ref.factors(R)
    for n in range(3):
        ref.set_Y(n, Y[n])
    ref.sweep_begin()
    p = d.Plan(dims, vals, idx, threads=T, rank=R)
    for n in range(3):
        p.set_factor(n, Y[n])
    for sweep, n in [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2)]:
        ref.process(n)
        p.process(n)
        gv, gi = p.slab()
        rv, ri = ref.slab()
        same = np.array_equal(gv.view(np.uint32), rv.view(np.uint32)) and \
            all(np.array_equal(a, b) for a, b in zip(gi, ri))
        ndiff = int(np.count_nonzero(gi[(n + 1) % 3] != ri[(n + 1) % 3]))
        if sweep == 1:
            print(f"\nsweep 1 mode {n}: slab {'bit-exact' if same else f'DIFFERS ({ndiff})'}")
            assert same, f"slab after the second sweep's process({n}) differs from the reference's"
            continue
        yg = p.yhat(n)[:, :R]
        yr = ref.yhat(n)[:, :R]
        y64 = refb.mttkrp_f64(vals, idx, n, Y, R, int(dims[n]))[:, :R]
        e64, eref, ref64 = rel_fro(yg, y64), rel_fro(yg, yr), rel_fro(yr, y64)
        print(f"\nmode {n}: slab {'bit-exact' if same else f'DIFFERS ({ndiff} next-mode indices)'}; "
              f"Yhat rel-Fro vs FP64 {e64:.2e}, vs reference {eref:.2e} "
              f"(reference vs FP64 {ref64:.2e})")
        assert same, f"slab after process({n}) differs from the reference's"
        assert e64 < 1e-5
        assert eref < max(1e-5, 2.0 * ref64)
    p.close()


# ---------------------------------------------------------------------------
#  4-mode mixed precision at full size: one GS and one Jacobi iteration
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def four_mode_full():
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.cp_zipf_torch((50_000, 20_000, 2_000, 500), 200_000_000,
                                          (0, 0, 1.3, 1.3), 10, 0.05, 3, "cuda")
    return np.asarray(dims, np.uint32), vals, idx


@pytest.mark.parametrize("kernel", ["gs", "jacobi"])
def test_four_mode_full_size_bf16_iteration_against_fp64(bindings, four_mode_full, kernel):
    """~200M nonzeros, rank 64, BF16 gathers, FP64 solves and fit: one
    iteration from the seed-42 initialisation.  The fit is within 1e-4 of
    FP64 CP-ALS; every factor is within 1e-2 of FP64 (the BF16 rounding of
    the gathered factors, ~2.6e-3 on a 2M-nonzero tensor of this shape) and
    within 1e-4 of the FP64 iteration whose MTTKRP reads BF16-rounded
    factors, the last mode's in FP32 (the rest is FP32 accumulation)."""
    import dynasor_plus_b200 as d
    dims, vals, idx = four_mode_full
    R = 64
    p = d.Plan(dims, vals, idx, threads=16, rank=R, precision="bf16")
    r = p.cpals(max_iters=1, tol=0.0, seed=42, kernel=kernel)
    Yg = [p.factor(n) for n in range(4)]
    p.close()
    jac = kernel == "jacobi"
    fit64, Y64, _ = bindings.cpals_f64(dims, vals, idx, R, 1, 0.0, seed=42, jacobi=jac)
    fitb, Yb, _ = bindings.cpals_f64(dims, vals, idx, R, 1, 0.0, seed=42, jacobi=jac,
                                     bf16_gathers=True, last_mode_fp32=True)
    e64 = [rel_fro(Yg[n][:, :R], Y64[n][:, :R]) for n in range(4)]
    eb = [rel_fro(Yg[n][:, :R], Yb[n][:, :R]) for n in range(4)]
    df = abs(r["fit_history"][0] - fit64[0])
    print(f"\n4-mode {len(vals)} nnz rank 64 BF16 {kernel}: fit {r['fit_history'][0]:.8f} "
          f"vs FP64 {fit64[0]:.8f} (|d| {df:.2e}); factor rel-Fro vs FP64 "
          + " ".join(f"{x:.2e}" for x in e64) + "; vs FP64 with BF16 gathers "
          + " ".join(f"{x:.2e}" for x in eb))
    assert df < FIT_TOL
    assert max(e64) < 1e-2
    assert max(eb) < 1e-4


# ---------------------------------------------------------------------------
#  CP-OPT gradient at full size
# ---------------------------------------------------------------------------
def test_cpopt_gradient_full_size(refb):
    """Gradient of 0.5 * ||X - M||^2 (dense model M) w.r.t. every factor on
    the 20M-nonzero tensor, rank 32, factors N(0, 0.1).

    Central differences (h = 1e-4, FP64) at 64 random entries: only the
    nonzeros in the perturbed row and the perturbed mode's Gram change, so
    f(Y +- h e) is evaluated from those terms in FP64 (the unchanged terms
    are the same numbers on both sides and cancel).  Then the whole gradient
    against one built from the reference's spmttkrp_reference:
    Y[n] * Hadamard(Grams) - MTTKRP_n."""
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((100_000, 100_000, 1_000), 20_000_000, seed=21,
                                    values="normal")
    R, Rp = 32, 32
    rng = np.random.default_rng(22)
    Y = [np.asarray(rng.normal(0, 0.1, (int(dn), Rp)), np.float32) for dn in dims]
    p = d.Plan(dims, vals, idx, threads=16, rank=R)
    for n in range(3):
        p.set_factor(n, Y[n])
    g = p.cpopt_gradient()
    p.close()
    Y64 = [y.astype(np.float64) for y in Y]
    G = [y.T @ y for y in Y64]
    x = vals.astype(np.float64)
    h = 1e-4
    worst = 0.0
    for _ in range(64):
        n = int(rng.integers(0, 3))
        i = int(rng.integers(0, int(dims[n])))
        r = int(rng.integers(0, R))
        sel = np.flatnonzero(idx[n] == i)
        others = [w for w in range(3) if w != n]
        prod = Y64[others[0]][idx[others[0]][sel]] * Y64[others[1]][idx[others[1]][sel]]
        P = G[others[0]] * G[others[1]]
        f = []
        for s in (h, -h):
            yi = Y64[n][i].copy()
            yi[r] += s
            inner = float(x[sel] @ (prod @ yi))            # <X, M> over the affected nonzeros
            Gn = G[n] - np.outer(Y64[n][i], Y64[n][i]) + np.outer(yi, yi)
            f.append(-inner + 0.5 * float((Gn * P).sum()))
        fd = (f[0] - f[1]) / (2 * h)
        worst = max(worst, abs(float(g[n][i, r]) - fd) / max(1.0, abs(fd)))
    ref = refb.Reference(dims, vals, idx)
    ref.build(16, "pingpong")
    ref.factors(R)
    for n in range(3):
        ref.set_Y(n, Y[n])
    ref.reference_mttkrp()
    errs = []
    for n in range(3):
        Hn = np.ones((R, R))
        for m in range(3):
            if m != n:
                Hn *= G[m]
        expect = Y64[n] @ Hn - ref.yhat(n)[:, :R]
        errs.append(rel_fro(g[n][:, :R], expect))
    print(f"\nCP-OPT gradient 20M nnz rank 32: worst FD rel error {worst:.2e}; "
          "vs reference-MTTKRP gradient " + " ".join(f"{e:.2e}" for e in errs))
    assert worst < 1e-3
    assert max(errs) < 1e-5


# ---------------------------------------------------------------------------
#  16 restarts x rank 16 on the 50M-draw Zipf(1.0) tensor
# ---------------------------------------------------------------------------
def test_restarts_full_size_against_fp64(bindings):
    """K = 16 restarts of rank 16 (effective rank 256) in one plan, 5
    Gauss-Seidel iterations; restarts 0, 7 and 15 against FP64 CP-ALS runs
    from seeds 42, 49 and 57."""
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.cp_zipf_torch((400_000, 300_000, 2_000), 50_000_000,
                                          (1.0, 1.0, 1.0), 8, 0.02, 4, "cuda")
    dims = np.asarray(dims, np.uint32)
    K, Re, it = 16, 16, 5
    p = d.Plan(dims, vals, idx, threads=16, rank=K * Re)
    res = p.cpals_multistart(K, max_iters=it, tol=0.0, seed=42)
    Yg = [p.factor(n) for n in range(3)]
    p.close()
    for k in (0, 7, 15):
        fit64, Y64, _ = bindings.cpals_f64(dims, vals, idx, Re, it, 0.0, seed=42 + k)
        df = float(np.max(np.abs(res[k]["fit_history"] - fit64)))
        ef = [rel_fro(Yg[n][:, k * Re:(k + 1) * Re], Y64[n][:, :Re]) for n in range(3)]
        print(f"\nrestart {k} ({len(vals)} nnz): max |dfit| {df:.2e}; factor rel-Fro "
              + " ".join(f"{e:.2e}" for e in ef))
        assert df < 1e-6
        assert max(ef) < 1e-3


# ---------------------------------------------------------------------------
#  32 tensors of uneven size in one batch
# ---------------------------------------------------------------------------
def test_tensor_batch_against_single_runs_and_fp64(bindings):
    """32 tensors (dims log-uniform in [1e3, 1e5] per mode, nnz log-uniform
    in [1e4, 5e6], rank-4 truth + 1% noise), rank 8, 30 iterations, tol 1e-4:
    every batched run equals a single run of the same plan options, and the
    largest and smallest tensors follow FP64 CP-ALS."""
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    ts = synth.tensor_batch(32, seed=17)
    plans = [d.Plan(dims, v, i, threads=16, rank=8) for dims, v, i in ts]
    batch = d.cpals_batch(plans, max_iters=30, tol=1e-4, seed=42)
    for pl in plans:
        pl.close()
    sizes = [len(v) for _, v, _ in ts]
    for k, (dims, v, i) in enumerate(ts):
        q = d.Plan(dims, v, i, threads=16, rank=8)
        r = q.cpals(max_iters=30, tol=1e-4, seed=42)
        q.close()
        assert batch[k]["iters_done"] == r["iters_done"]
        assert np.max(np.abs(batch[k]["fit_history"] - r["fit_history"])) < 1e-6
    for k in (int(np.argmax(sizes)), int(np.argmin(sizes))):
        dims, v, i = ts[k]
        fit64, _, _ = bindings.cpals_f64(dims, v, i, 8, 30, 1e-4, seed=42)
        h = batch[k]["fit_history"]
        m = min(len(h), len(fit64))
        df = float(np.max(np.abs(h[:m] - fit64[:m])))
        print(f"\nbatch tensor {k} ({sizes[k]} nnz): iters {len(h)} / fp64 {len(fit64)}, "
              f"max |dfit| {df:.2e}")
        assert len(h) == len(fit64)
        assert df < 1e-6
