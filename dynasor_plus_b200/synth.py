"""Seeded synthetic sparse tensors with the shapes and value distributions of
the benchmark workloads (no dataset files are used anywhere).

All generators return ``(dims, vals, idx)``: ``dims`` uint32[N], ``vals``
float32[nnz], ``idx`` a list of N uint32[nnz] arrays with 0-based indices.

* ``uniform``       uniform coordinates, U(-1,1) values, duplicates kept (the
                    layout of a random .tns; duplicates are legal input).
* ``cp_truth``      3-mode rank-5 CP model with U(0,1) factors at distinct
                    uniform coordinates plus N(0, (1% mean)^2) noise
                    (the 200^3 / 100k-nonzero CP-ALS workload).
* ``tensor_batch``  many small 3-mode CP-model tensors of uneven size: dims
                    log-uniform per mode, nnz log-uniform (the 32-tensor
                    batch workload: [1e3, 1e5] per mode, [1e4, 5e6] nnz).
* ``zipf``          per-mode Zipf(s) coordinates over a seed-permuted index
                    set, duplicates merged, LogNormal(0,1) values (the
                    1,000,000 x 200,000 x 50,000 MTTKRP workload when called
                    with 100M draws).  A torch/GPU variant generates the full
                    size in well under a second on a B200.
"""
from __future__ import annotations

import numpy as np


def uniform(dims, nnz, seed=0, values="uniform"):
    rng = np.random.default_rng(seed)
    dims = np.asarray(dims, np.uint32)
    idx = [rng.integers(0, int(d), size=nnz, dtype=np.int64).astype(np.uint32) for d in dims]
    if values == "normal":
        vals = rng.standard_normal(nnz).astype(np.float32)
    else:
        vals = rng.uniform(-1.0, 1.0, nnz).astype(np.float32)
    return dims, vals, idx


def _distinct_linear(rng, dims, nnz):
    total = int(np.prod(np.asarray(dims, np.float64)))
    if nnz > total:
        raise ValueError("more nonzeros than cells")
    if total <= 50_000_000:
        lin = rng.choice(total, nnz, replace=False)
    else:
        lin = np.unique(rng.integers(0, total, size=int(nnz * 1.05) + 16, dtype=np.int64))
        while lin.size < nnz:
            extra = rng.integers(0, total, size=nnz, dtype=np.int64)
            lin = np.unique(np.concatenate([lin, extra]))
        lin = rng.permutation(lin)[:nnz]
    return np.stack(np.unravel_index(lin, tuple(int(d) for d in dims)), 1)


def cp_truth(dims=(200, 200, 200), nnz=100_000, rank=5, noise=0.01, seed=1, factor="uniform"):
    """Values = CP model (rank `rank`, factors U(0,1) or |N(0,1)|) at distinct
    uniform coordinates + Gaussian noise with sigma = noise * mean value."""
    rng = np.random.default_rng(seed)
    dims = np.asarray(dims, np.uint32)
    if factor == "uniform":
        U = [rng.uniform(0, 1, (int(d), rank)) for d in dims]
    else:
        U = [np.abs(rng.standard_normal((int(d), rank))) for d in dims]
    coords = _distinct_linear(rng, dims, nnz)
    v = np.ones((nnz, rank))
    for n in range(len(dims)):
        v *= U[n][coords[:, n]]
    v = v.sum(1)
    v = v + rng.normal(0.0, noise * v.mean(), nnz)
    idx = [np.ascontiguousarray(coords[:, n], np.uint32) for n in range(len(dims))]
    return dims, v.astype(np.float32), idx


def tensor_batch(count=32, seed=17, dim_range=(1_000, 100_000), nnz_range=(10_000, 5_000_000),
                 rank=4, noise=0.01):
    """`count` independent ``cp_truth`` tensors (rank-`rank` U(0,1) truth plus
    `noise` relative Gaussian noise), each with three mode sizes drawn
    log-uniform in `dim_range` and a nonzero count drawn log-uniform in
    `nnz_range`.  Returns a list of (dims, vals, idx)."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(dim_range[0]), np.log(dim_range[1])
    nlo, nhi = np.log(nnz_range[0]), np.log(nnz_range[1])
    out = []
    for k in range(count):
        dims = tuple(int(x) for x in np.exp(rng.uniform(lo, hi, 3)))
        nnz = int(np.exp(rng.uniform(nlo, nhi)))
        out.append(cp_truth(dims, nnz, rank, noise, seed=int(rng.integers(0, 2**31))))
    return out


def _zipf_cdf(I, s):
    p = 1.0 / np.arange(1, I + 1, dtype=np.float64) ** s
    c = np.cumsum(p)
    return c / c[-1]


def zipf(dims=(1_000_000, 200_000, 50_000), draws=1_000_000, s=1.1, seed=2):
    """Zipf(s) coordinates per mode over a seed-permuted index set, merged
    duplicates, LogNormal(0,1) values.  `s` may be a per-mode sequence; an
    entry of 0 means uniform coordinates for that mode."""
    rng = np.random.default_rng(seed)
    dims = np.asarray(dims, np.uint32)
    N = len(dims)
    ss = list(s) if np.ndim(s) else [s] * N
    cols = []
    for n in range(N):
        I = int(dims[n])
        if ss[n] == 0:
            cols.append(rng.integers(0, I, size=draws, dtype=np.int64))
            continue
        perm = rng.permutation(I)
        u = rng.random(draws)
        k = np.searchsorted(_zipf_cdf(I, ss[n]), u, side="right")
        cols.append(perm[np.minimum(k, I - 1)])
    lin = np.zeros(draws, np.int64)
    for n in range(N):
        lin = lin * int(dims[n]) + cols[n]
    lin = np.unique(lin)
    coords = np.stack(np.unravel_index(lin, tuple(int(d) for d in dims)), 1)
    vals = rng.lognormal(0.0, 1.0, lin.size).astype(np.float32)
    idx = [np.ascontiguousarray(coords[:, n], np.uint32) for n in range(N)]
    return dims, vals, idx


def zipf_torch(dims=(1_000_000, 200_000, 50_000), draws=100_000_000, s=1.1, seed=2,
               device="cuda"):
    """GPU variant of ``zipf`` (same distribution, torch RNG): inverse-CDF
    sampling with searchsorted, duplicates merged with torch.unique.
    Returns host numpy arrays like the other generators."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    dims_l = [int(d) for d in dims]
    N = len(dims_l)
    ss = list(s) if np.ndim(s) else [s] * N
    lin = torch.zeros(draws, dtype=torch.int64, device=device)
    for n in range(N):
        I = dims_l[n]
        if ss[n] == 0:
            col = torch.randint(0, I, (draws,), generator=g, device=device)
        else:
            cdf = torch.from_numpy(_zipf_cdf(I, ss[n])).to(device)
            perm = torch.randperm(I, generator=g, device=device)
            u = torch.rand(draws, generator=g, device=device, dtype=torch.float64)
            k = torch.searchsorted(cdf, u, right=True).clamp_(max=I - 1)
            col = perm[k]
            del cdf, u, k
        lin = lin * I + col
        del col
    lin = torch.unique(lin)
    nnz = lin.numel()
    idx = []
    rem = lin
    for n in reversed(range(N)):
        idx.append((rem % dims_l[n]).to(torch.int32))
        rem = rem // dims_l[n]
    idx = idx[::-1]
    vals = torch.empty(nnz, device=device, dtype=torch.float32).log_normal_(0.0, 1.0, generator=g)
    out_idx = [i.cpu().numpy().view(np.uint32) for i in idx]
    return np.asarray(dims_l, np.uint32), vals.cpu().numpy(), out_idx


def cp_zipf_torch(dims=(50_000, 20_000, 2_000, 500), draws=200_000_000, s=(0, 0, 1.3, 1.3),
                  rank=10, noise=0.05, seed=3, device="cuda"):
    """Coordinates as ``zipf_torch`` (per-mode Zipf exponents, 0 = uniform),
    values from a rank-`rank` CP model with |N(0,1)| factors plus Gaussian
    noise with sigma = `noise` x mean value (the 4-mode mixed-precision
    CP-ALS workload).  Returns host numpy arrays."""
    import torch

    dims, _, idx = zipf_torch(dims, draws, s, seed, device)
    g = torch.Generator(device=device)
    g.manual_seed(seed + 7)
    U = [torch.randn((int(I), rank), generator=g, device=device).abs_() for I in dims]
    v = None
    for r in range(rank):
        t = None
        for n in range(len(dims)):
            ix = torch.from_numpy(idx[n].view(np.int32)).to(device).long()
            col = U[n][:, r][ix]
            del ix
            t = col if t is None else t * col
        v = t if v is None else v + t
    v = v + torch.randn(v.numel(), generator=g, device=device) * (noise * v.mean())
    return dims, v.float().cpu().numpy(), idx
