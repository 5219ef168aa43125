"""Owner-computes CP-ALS over several GPUs: one process per GPU,
torch.distributed for the collectives (NCCL on GPUs).

The reference partitions the output rows of every mode by owner
(src/dynasor.cpp:8-20: each worker owns super-shards, so a row of Yhat[n]
has exactly one writer).  Across GPUs the same idea gives:

* every rank owns one contiguous block of rows of every mode, the blocks
  chosen so each holds about the same number of nonzeros (rows are cut where
  the running nonzero count crosses k/G of the total);
* for mode n a rank keeps the nonzeros whose mode-n index falls in its
  block, as an NCopy plan of the engine (so the MTTKRP needs no exchange of
  nonzeros, ever: the tensor is distributed once, by mode);
* the factors are replicated: after a rank updates the rows of its block, an
  all-gather rebuilds Y[n] everywhere; the R x R Gram of Y[n] is an
  all-reduce of the block Grams (FP64); the column norms and the fit's two
  sums are all-reduces of a few numbers.

Per mode and iteration the wire carries I_n x Rp x 4 bytes (the all-gather)
plus R^2 x 8 and R x 8 bytes: the MTTKRP (the engine's row-run kernel on the
rank's nonzeros) and the factor update of the rank's rows are the work that
shrinks with the number of ranks.  The update follows the single-GPU one in
arithmetic: FP64 Hadamard of Grams with the reference's relative ridge, a
Cholesky whose non-positive pivots give zero components
(src/dynasor_linalg.cpp:160-246) turned into an R x R map on the host, the
rows mapped by one FP64 GEMM, FP64 column norms.

`local_mttkrp` is the hook that computes a rank's MTTKRP rows; the default
(`EngineMttkrp`) runs the engine on the rank's GPU.  Tests on machines
without a GPU pass a CPU stand-in to check the partitioning and the
collectives over gloo ranks.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import Plan, init_factor, padded_rank


def row_blocks(counts, parts: int):
    """Boundaries b[0] = 0 <= ... <= b[parts] = len(counts) of `parts`
    contiguous row blocks with about equal nonzero counts: block k ends
    after the first row where the running count reaches (k+1)/parts of the
    total."""
    counts = np.asarray(counts, np.int64)
    rows = len(counts)
    cum = np.cumsum(counts)
    total = int(cum[-1]) if rows else 0
    b = [0]
    for k in range(1, parts):
        if total == 0:
            cut = rows * k // parts
        else:
            cut = int(np.searchsorted(cum, total * k / parts, side="left")) + 1
        b.append(min(rows, max(b[-1], cut)))
    b.append(rows)
    return b


class _DeviceArray:
    """A device buffer described by __cuda_array_interface__ (zero-copy
    torch view of a plan's factor memory)."""

    def __init__(self, ptr: int, shape, typestr="<f4"):
        self.__cuda_array_interface__ = {"shape": tuple(int(s) for s in shape),
                                         "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class EngineMttkrp:
    """A rank's MTTKRP rows of every mode on its GPU: for mode n, an NCopy
    plan of the nonzeros whose mode-n index lies in the rank's block (the
    other indices keep their global values, so the plan gathers the
    replicated factors directly).  Factors are copied device to device into
    the plan before each mode; everything runs on torch's current stream."""

    def __init__(self, dims, vals, idx, blocks, me, rank, threads, device):
        import torch
        self.torch = torch
        self.N = len(dims)
        self.R, self.Rp = int(rank), padded_rank(rank)
        self.blocks = blocks
        self.me = me
        self.plans, self.Yv, self.Yhv = [], [], []
        stream = torch.cuda.current_stream(device)
        for n in range(self.N):
            lo, hi = blocks[n][me], blocks[n][me + 1]
            sel = np.flatnonzero((idx[n] >= lo) & (idx[n] < hi))
            p = None
            if sel.size:
                p = Plan(dims, vals[sel], [i[sel] for i in idx], threads=threads, rank=rank,
                         layout="ncopy", device=device.index if device.index is not None else 0)
                p.set_stream(stream)
            self.plans.append(p)
            views, hv = [], None
            if p is not None:
                for w in range(self.N):
                    y, yh = p.device_ptrs(w)
                    views.append(torch.as_tensor(_DeviceArray(y, (int(dims[w]), self.Rp)),
                                                 device=device))
                    if w == n:
                        hv = torch.as_tensor(_DeviceArray(yh, (int(dims[w]), self.Rp)),
                                             device=device)
            self.Yv.append(views)
            self.Yhv.append(hv)

    def __call__(self, n, Y):
        lo, hi = self.blocks[n][self.me], self.blocks[n][self.me + 1]
        p = self.plans[n]
        if p is None:
            return self.torch.zeros((hi - lo, self.Rp), dtype=self.torch.float32, device=Y[0].device)
        for w in range(self.N):
            if w != n:
                self.Yv[n][w].copy_(Y[w])
        p.process(n)
        return self.Yhv[n][lo:hi]

    def close(self):
        for p in self.plans:
            if p is not None:
                p.close()


def _solve_map(V, ridge):
    """R x R map W with Y = Yhat W: Cholesky of V + ridge * max(diag V) * I,
    non-positive pivots clamped to zero and their components set to zero,
    forward then backward substitution per row (the reference's la::
    cholesky_lower / right_solve_chol semantics), built on the host in FP64
    by solving the rows of the identity."""
    R = V.shape[0]
    A = V.copy()
    A[np.diag_indices(R)] += max(ridge * float(np.max(np.diag(V))), 0.0)
    L = np.zeros((R, R))
    for j in range(R):
        s = A[j, j] - L[j, :j] @ L[j, :j]
        d = math.sqrt(s) if s > 0 else 0.0
        L[j, j] = d
        inv = 1.0 / d if d > 0 else 0.0
        L[j + 1:, j] = (A[j + 1:, j] - L[j + 1:, :j] @ L[j, :j]) * inv
    X = np.eye(R)
    for r in range(R):                          # forward: L y = b
        d = L[r, r]
        X[:, r] = (X[:, r] - X[:, :r] @ L[r, :r]) / d if d > 0 else 0.0
    for r in range(R - 1, -1, -1):              # backward: L^T x = y
        d = L[r, r]
        X[:, r] = (X[:, r] - X[:, r + 1:] @ L[r + 1:, r]) / d if d > 0 else 0.0
    return X                                     # row i of X = solve(e_i): Y = Yhat @ X


class OwnerComputesCpals:
    """CP-ALS (Gauss-Seidel) with the rows of every mode split over the
    ranks of `group`.  Every rank passes the same COO tensor; each keeps only
    the nonzeros of its row blocks.  Results (fits, factors, lambda) are the
    same on every rank."""

    def __init__(self, dims, vals, idx, rank, threads=16, group=None, device=None,
                 local_mttkrp=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group
        self.ws = dist.get_world_size(group) if dist.is_initialized() else 1
        self.me = dist.get_rank(group) if dist.is_initialized() else 0
        self.dims = np.asarray(dims, np.uint32)
        self.N = len(dims)
        self.R, self.Rp = int(rank), padded_rank(rank)
        idx = [np.ascontiguousarray(i, np.uint32) for i in idx]
        vals = np.ascontiguousarray(vals, np.float32)
        self.blocks = [row_blocks(np.bincount(idx[n], minlength=int(dims[n])), self.ws)
                       for n in range(self.N)]
        self.device = torch.device(device) if device is not None else (
            torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available()
            else torch.device("cpu"))
        if local_mttkrp is None:
            local_mttkrp = EngineMttkrp(dims, vals, idx, self.blocks, self.me, rank, threads,
                                        self.device)
        self.mttkrp = local_mttkrp
        # gloo collectives take host tensors: device tensors are staged
        # through host memory for them (NCCL takes device tensors as they are)
        self.stage = (self.ws > 1 and self.device.type == "cuda"
                      and dist.get_backend(group) == "gloo")
        lo, hi = self.blocks[self.N - 1][self.me], self.blocks[self.N - 1][self.me + 1]
        mine = (idx[self.N - 1] >= lo) & (idx[self.N - 1] < hi)
        v = vals[mine].astype(np.float64)
        self.tn2 = self._sum(float(v @ v))

    # -- collectives -----------------------------------------------------
    def _allreduce(self, t):
        if self.ws > 1:
            if self.stage and t.is_cuda:
                h = t.cpu()
                self.dist.all_reduce(h, group=self.group)
                t.copy_(h)
            else:
                self.dist.all_reduce(t, group=self.group)
        return t

    def _sum(self, x: float) -> float:
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        return float(self._allreduce(t).item())

    def _allgather_rows(self, n, blk):
        """The full I_n x Rp factor from every rank's block of rows."""
        torch = self.torch
        if self.ws == 1:
            return blk.contiguous()
        b = self.blocks[n]
        mx = max(b[k + 1] - b[k] for k in range(self.ws))
        pad = torch.zeros((mx, self.Rp), dtype=blk.dtype, device=blk.device)
        pad[:blk.shape[0]] = blk
        if self.stage and pad.is_cuda:
            out = torch.empty((self.ws * mx, self.Rp), dtype=blk.dtype)
            self.dist.all_gather_into_tensor(out, pad.cpu(), group=self.group)
            out = out.to(blk.device)
        else:
            out = torch.empty((self.ws * mx, self.Rp), dtype=blk.dtype, device=blk.device)
            self.dist.all_gather_into_tensor(out, pad, group=self.group)
        return torch.cat([out[k * mx:k * mx + b[k + 1] - b[k]] for k in range(self.ws)])

    # -- the run ---------------------------------------------------------
    def run(self, max_iters=50, tol=1e-4, seed=42, ridge=1e-10, init=None):
        torch = self.torch
        N, R, Rp, dev = self.N, self.R, self.Rp, self.device
        t0 = time.time()
        if init is None:
            # mode 0's initial factor is never read by Gauss-Seidel (it is
            # solved first from the other modes' Grams): zero instead of drawn
            Y = [torch.zeros((int(self.dims[0]), Rp), dtype=torch.float32, device=dev)] + [
                torch.from_numpy(init_factor(seed, n, int(self.dims[n]), R)).to(dev)
                for n in range(1, N)]
        else:
            Y = [torch.as_tensor(np.asarray(y, np.float32)).to(dev) for y in init]
        G = [Y[n][:, :R].double().T @ Y[n][:, :R].double() for n in range(N)]
        lam = torch.ones(R, dtype=torch.float64, device=dev)
        fits, fit_prev = [], 0.0
        for it in range(max_iters):
            for n in range(N):
                lo, hi = self.blocks[n][self.me], self.blocks[n][self.me + 1]
                yh = self.mttkrp(n, Y)                        # rows [lo, hi) x Rp
                V = torch.ones((R, R), dtype=torch.float64, device=dev)
                for m in range(N):
                    if m != n:
                        V = V * G[m]
                W = torch.from_numpy(_solve_map(V.cpu().numpy(), ridge)).to(dev)
                blk = yh[:, :R].double() @ W                  # the rank's rows, FP64
                nrm = self._allreduce((blk * blk).sum(0))
                lam = torch.sqrt(nrm)
                inv = torch.where(lam > 1e-20, 1.0 / lam, torch.zeros_like(lam))
                blk = blk * inv
                full = torch.zeros((hi - lo, Rp), dtype=torch.float32, device=dev)
                full[:, :R] = blk.float()
                Y[n] = self._allgather_rows(n, full)
                G[n] = self._allreduce(blk.T @ blk)
                if n == N - 1:
                    inner = self._allreduce((lam * (blk * yh[:, :R].double()).sum(0)).sum()
                                            .reshape(1)).item()
            m2 = torch.ones((R, R), dtype=torch.float64, device=dev)
            for n in range(N):
                m2 = m2 * G[n]
            m2 = float((lam[:, None] * lam[None, :] * m2).sum().item())
            res2 = max(0.0, self.tn2 - 2.0 * inner + max(0.0, m2))
            fit = 1.0 - math.sqrt(res2) / max(math.sqrt(self.tn2), 1e-30)
            fits.append(fit)
            if it > 0 and abs(fit - fit_prev) < tol:
                break
            fit_prev = fit
        if dev.type == "cuda":
            torch.cuda.synchronize(dev)
        return {"iters_done": len(fits), "fit_history": np.asarray(fits),
                "final_fit": fits[-1] if fits else 0.0, "lambda": lam.cpu().numpy(),
                "factors": [y.cpu().numpy() for y in Y], "total_time_s": time.time() - t0}

    def close(self):
        close = getattr(self.mttkrp, "close", None)
        if close:
            close()
