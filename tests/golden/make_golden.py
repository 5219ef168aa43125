"""Regenerate the golden fixtures of tests/golden/ from the reference itself.

    python tests/golden/make_golden.py --ref <reference tree>   (or REF=<tree>)

Drives the UNMODIFIED reference sources compiled by oracle/Makefile
(oracle/_ref/libdynref_*.so) through their own API -- build_flycoo,
SpmttkrpSweep::process, spmttkrp_reference, cpals -- and stores, per case:

  dims, vals, idx{n}            the input COO (0-based)
  shift, K, kclass              plan geometry
  sbeg{n}, send{n}              shard ranges
  sched_counts{n}, sched{n}     LPT schedule (per-worker counts + flat list)
  cursors{n}                    the reference's remap cursor table
  slab0_v, slab0_i{n}           slab after build_flycoo (mode-0 order)
  slab_s{s}_m{n}_v / _i{k}      slab after process(n) of sweep s
  Y{n}                          U(0,1) --verify factors (seed 42)
  yhat_s{s}_m{n}                Yhat[n] of sweep s (reference FP32)
  yref{n}                       spmttkrp_reference (single thread) output

plus a CP-ALS case (fit history of cpals, Gauss-Seidel, seed 42).  The
fixtures are small so the oracle can be pinned on any machine, including
one without the reference tree.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import bindings as B  # noqa: E402
from dynasor_plus_b200 import synth  # noqa: E402


def read_tns(path):
    rows = []
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t or t[0].startswith("#"):
                continue
            rows.append([float(x) for x in t])
    a = np.array(rows)
    N = a.shape[1] - 1
    idx = [(a[:, n].astype(np.int64) - 1).astype(np.uint32) for n in range(N)]
    dims = np.array([int(i.max()) + 1 for i in idx], np.uint32)
    return dims, a[:, N].astype(np.float32), idx


def sweep_case(dims, vals, idx, T, R, fiber, sweeps=2):
    out = {"dims": dims, "vals": vals, "T": np.array(T), "R": np.array(R),
           "fiber": np.array(int(fiber))}
    N = len(dims)
    for n in range(N):
        out[f"idx{n}"] = idx[n]
    ref = B.Reference(dims, vals, idx)
    ref.build(T, "pingpong")
    out["shift"], out["K"], out["kclass"] = ref.shift, ref.K, ref.kclass
    for n in range(N):
        out[f"sbeg{n}"], out[f"send{n}"] = ref.shards(n)
        out[f"sched_counts{n}"], out[f"sched{n}"] = ref.schedule(n)
        out[f"cursors{n}"] = ref.cursors(n)
    v, ix = ref.slab()
    out["slab0_v"] = v
    for n in range(N):
        out[f"slab0_i{n}"] = ix[n]
    ref.factors(R)
    Y = B.uniform_factors(42, dims, R)
    for n in range(N):
        ref.set_Y(n, Y[n])
        out[f"Y{n}"] = Y[n]
    ref.sweep_begin(fiber_off=not fiber)
    for s in range(sweeps):
        for n in range(N):
            ref.process(n)
            out[f"yhat_s{s}_m{n}"] = ref.yhat(n)
            v, ix = ref.slab()
            out[f"slab_s{s}_m{n}_v"] = v
            for k in range(N):
                out[f"slab_s{s}_m{n}_i{k}"] = ix[k]
    ref.reference_mttkrp()
    for n in range(N):
        out[f"yref{n}"] = ref.yhat(n)
    return out


def cpals_case(dims, vals, idx, T, R, iters, tol):
    ref = B.Reference(dims, vals, idx)
    ref.build(T, "pingpong")
    fit, lam, _, _ = ref.cpals(R, iters, tol, seed=42)
    out = {"dims": dims, "vals": vals, "T": np.array(T), "R": np.array(R),
           "iters": np.array(iters), "tol": np.array(tol), "fit": fit, "lam": lam}
    for n in range(len(dims)):
        out[f"idx{n}"] = idx[n]
        out[f"Y{n}"] = ref.get_Y(n)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("REF"), required="REF" not in os.environ,
                    help="the reference source tree (or set REF)")
    a = ap.parse_args()
    if not B.ref_available():
        sys.exit("oracle/_ref is not built; run `make -C oracle ref` first")

    cases = {}
    d7 = read_tns(os.path.join(a.ref, "data", "3d_7.tns"))
    cases["ref_3d7_T2_R16.npz"] = sweep_case(*d7, T=2, R=16, fiber=True)
    cases["ref_3d7_T1_R8.npz"] = sweep_case(*d7, T=1, R=8, fiber=True)
    cases["ref_rand3d_T4_R16_fiber.npz"] = sweep_case(
        *synth.uniform((64, 48, 24), 3000, seed=11), T=4, R=16, fiber=True)
    cases["ref_rand3d_T4_R16_nofiber.npz"] = sweep_case(
        *synth.uniform((64, 48, 24), 3000, seed=11), T=4, R=16, fiber=False)
    cases["ref_rand4d_T3_R20.npz"] = sweep_case(
        *synth.uniform((40, 30, 20, 10), 2500, seed=12), T=3, R=20, fiber=True)
    cases["ref_zipf3d_T8_R16.npz"] = sweep_case(
        *synth.zipf((1500, 300, 120), draws=8000, s=1.1, seed=13), T=8, R=16, fiber=True,
        sweeps=1)
    cases["ref_cpals_r5.npz"] = cpals_case(
        *synth.cp_truth((20, 25, 30), 4000, rank=5, seed=7), T=2, R=5, iters=15, tol=0.0)
    for name, d in cases.items():
        np.savez_compressed(os.path.join(HERE, name), **d)
        print(name, os.path.getsize(os.path.join(HERE, name)), "bytes")


if __name__ == "__main__":
    main()
