"""Benchmark: mode-n sparse MTTKRP with the device remap on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (default): the skewed 3-mode MTTKRP tensor -- dims 1,000,000 x
200,000 x 50,000, 100M Zipf(s=1.1) coordinate draws per mode over a
seed-permuted index set, duplicates merged (~64.7M nonzeros), LogNormal(0,1)
values, rank 32 -- generated from a fixed seed (synthetic data, no files).

One step = one full MTTKRP sweep (modes 0,1,2 in order; each mode computes
Yhat[n] and remaps the slab for the next mode on the device).  `value` is
GNNZ/s in the reference's convention nnz / t_sweep (src/main.cpp:970-972),
over all ranks; `per_mode_gnnz_s` is nnz / t_mode.  Inputs stay resident
(the slab is 1 GB, far larger than the 126 MB L2, so no L2 flush is needed).

`e2e` is the same metric through the public host API
(dgpu_mttkrp_sweep_host): every step uploads the factor matrices from pinned
host memory, runs the sweep and downloads every Yhat.

Multi-GPU: replicas only (each rank runs its own copy of the workload, no
collective on the data path); value = total nnz processed / max-over-ranks
time, scaling "weak".

--impl reference times the reference's own CPU implementation (the
reference sources compiled into oracle/_ref) on this host's cores, on the
same workload and metric: one PingPong sweep of the whole tensor per step.
`cpu_baseline` is the same reference on the whole tensor, median of
--cpu-sweeps sweeps.

Beside the headline the line carries, each measured on its own workload:
`cpals` / `cpals_small` (CP-ALS iterations/s on this tensor and on the
200^3 / 100k-nonzero rank-16 configuration), `ncopy` (the NCopy layout),
`bf16` (4-mode 50,000 x 20,000 x 2,000 x 500 from 200M draws, rank 64:
CP-ALS iterations/s with FP32 and with BF16 gathers), `cpopt` (forward and
gradient on 100,000 x 100,000 x 1,000 with 20M nonzeros, rank 32) and
`batched` (16 restarts of rank 16 in one plan; 32 tensors in one batch;
each against the same runs one by one).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DIMS = (1_000_000, 200_000, 50_000)
DRAWS = 100_000_000
ZIPF_S = 1.1
SEED = 2
RANK = 32
METRIC = "MTTKRP GNNZ/s (nnz per full 3-mode sweep with device remap)"

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch,
# measured by ncu on this workload at its full size (64,659,576 nnz; one-pass
# metrics): profiles/k_part_replay_zipf1.1_64.7M.md (the partition passes of a
# sweep past the slab's first cycle, replayed) and
# profiles/dram_traffic_zipf1.1_64.7M.md (the MTTKRP).  Averages over one
# sweep's launches of each kind; scaled by nnz only when the bench runs
# another size.
NCU_NNZ = 64_659_576
NCU_DRAM_BYTES_PER_LAUNCH = {
    "part_scatter": 2_168_673_365,     # k_part_replay, the 3 remap passes
    "fiber_scatter": 2_169_593_941,    # k_part_replay, the 6 fiber-sort passes
    "mttkrp": 2_015_217_408,           # k_mttkrp_rowrun, 3 modes (1.57 / 2.06 / 2.41 GB)
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 150 on the GPU, so the timed region spans several 200 ms clock samples; 20 reference sweeps)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--threads", type=int, default=16,
                    help="plan worker count: the FLYCOO geometry of the reference run with "
                         "this many threads (16 = the GPU host's cores)")
    ap.add_argument("--layout", default="pingpong", choices=["pingpong", "ncopy", "auto"])
    ap.add_argument("--fiber", type=int, default=1)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "bf16"])
    ap.add_argument("--draws", type=int, default=DRAWS)
    ap.add_argument("--rank", type=int, default=RANK)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ncopy", action="store_true", help="skip the NCopy-layout line")
    ap.add_argument("--cpu-sweeps", type=int, default=2,
                    help="timed reference sweeps of the whole tensor in the CPU-baseline leg")
    ap.add_argument("--cpals-iters", type=int, default=5)
    ap.add_argument("--no-bf16", action="store_true",
                    help="skip the BF16-gather CP-ALS block (4-mode rank-64 tensor)")
    ap.add_argument("--bf16-draws", type=int, default=200_000_000,
                    help="coordinate draws of the 4-mode tensor of the BF16 block")
    ap.add_argument("--bf16-sweeps", type=int, default=2,
                    help="timed plain sweeps per plan of the BF16 block (launched from the host)")
    ap.add_argument("--no-cpopt", action="store_true",
                    help="skip the CP-OPT forward / gradient block (20M-nonzero tensor)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched blocks (16 restarts; 32 tensors)")
    ap.add_argument("--json-out", default=None)
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 20 if args.impl == "reference" else 150
    return args


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


CLOCK_REASONS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]


def summarize_clocks(lines, t0=None, t1=None):
    """Median SM clock, max clock and active throttle reasons of the
    nvidia-smi samples `lines` ((monotonic time, csv line) pairs) taken
    inside the timed region [t0, t1]; when the region is shorter than the
    sampling period and holds none, the first sample after t0 stands in."""
    parsed = []
    for t, line in lines:
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9:
            continue
        try:
            sm, smax = float(f[1]), float(f[2])
        except ValueError:
            continue
        rs = {nm for k, nm in enumerate(CLOCK_REASONS) if f[5 + k].lower().startswith("active")}
        parsed.append((t, sm, smax, rs))
    if not parsed:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
    sel = parsed
    if t0 is not None and t1 is not None:
        sel = [x for x in parsed if t0 <= x[0] <= t1]
        if not sel:
            sel = [x for x in parsed if x[0] >= t0][:1] or parsed[-1:]
    reasons = set()
    for x in sel:
        reasons |= x[3]
    out = {"sm_mhz": statistics.median(x[1] for x in sel),
           "sm_max_mhz": max(x[2] for x in sel),
           "reasons": sorted(reasons), "samples": len(sel), "samples_total": len(parsed)}
    if t0 is not None and t1 is not None:
        out["timed_region_s"] = round(t1 - t0, 3)
    return out


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms, read by a
    thread as they arrive; `start` returns once the first sample is in, and
    `begin`/`end` mark the timed region the summary keeps."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.thread = None
        self.lines = []
        self.t0 = self.t1 = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line))

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, bufsize=1)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        deadline = time.monotonic() + 5.0
        while not self.lines and self.proc.poll() is None and time.monotonic() < deadline:
            time.sleep(0.01)

    def begin(self):
        self.t0 = time.monotonic()

    def end(self):
        self.t1 = time.monotonic()

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)
        return summarize_clocks(list(self.lines), self.t0, self.t1)


def make_workload(args, device="cuda"):
    from dynasor_plus_b200 import synth
    if device == "cuda":
        return synth.zipf_torch(DIMS, args.draws, ZIPF_S, SEED, device="cuda")
    return synth.zipf(DIMS, args.draws, ZIPF_S, SEED)


def cpals_small_workload():
    """The plain CP-ALS configuration: 200 x 200 x 200, 100,000 distinct
    uniform coordinates, rank-5 U(0,1) truth + 1% Gaussian noise; rank 16,
    50 Gauss-Seidel iterations, tol 1e-4, seed 42 (synthetic, seeded)."""
    from dynasor_plus_b200 import synth
    return synth.cp_truth((200, 200, 200), 100_000, 5, 0.01, seed=1)


def cpals_small_gpu(threads):
    """CP-ALS iterations/s on the small configuration, both layouts."""
    import dynasor_plus_b200 as d
    dims, vals, idx = cpals_small_workload()
    out = {}
    for layout in ("ncopy", "pingpong"):
        p = d.Plan(dims, vals, idx, threads=threads, rank=16, layout=layout)
        p.cpals(max_iters=50, tol=1e-4, seed=42)          # warm-up
        r = p.cpals(max_iters=50, tol=1e-4, seed=42)
        out[layout] = {"iters": r["iters_done"], "iter_per_s": r["iters_done"] / r["total_time_s"],
                       "final_fit": r["final_fit"]}
        p.close()
    return out


def cpals_small_reference(threads):
    from oracle import bindings as B
    dims, vals, idx = cpals_small_workload()
    out = {}
    for layout in ("ncopy", "pingpong"):
        ref = B.Reference(dims, vals, idx)
        ref.build(threads, layout)
        fit, lam, tot, mt = ref.cpals(16, 50, 1e-4, 42)
        out[layout] = {"iters": len(fit), "iter_per_s": len(fit) / tot, "final_fit": float(fit[-1])}
    return out


def bf16_block(device, stream, args):
    """CP-ALS iterations/s with FP32 and with BF16 gathers (FP32 master
    factors, FP32 accumulation, FP64 solves and fit) on the 4-mode
    mixed-precision tensor: 50,000 x 20,000 x 2,000 x 500 from 200M draws
    (uniform modes 1-2, Zipf(1.3) modes 3-4), rank-10 |N(0,1)| truth + 5%
    noise, rank 64, Gauss-Seidel, both layouts.  Each timed run follows a
    warm-up run on the same plan; fits of the two precisions are compared
    iteration by iteration (their distance from FP64 CP-ALS is checked in
    tests/test_gpu_configs.py).  Each plan then times plain sweeps, every
    mode gathering in its precision (`--bf16-sweeps`)."""
    import torch
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.cp_zipf_torch((50_000, 20_000, 2_000, 500), args.bf16_draws,
                                          (0, 0, 1.3, 1.3), 10, 0.05, 3, "cuda")
    it = args.cpals_iters
    out = {"workload": f"4-mode 50000x20000x2000x500, {args.bf16_draws} draws deduped to "
                       f"{len(vals)} nnz, rank 64, GS, FP64 solve", "iters": it}
    for layout in ("ncopy", "pingpong"):
        res = {}
        sweep_ms = {}
        for prec in ("fp32", "bf16"):
            p = d.Plan(dims, vals, idx, threads=args.threads, rank=64, layout=layout,
                       precision=prec, device=device)
            p.set_stream(stream)
            p.cpals(max_iters=it, tol=0.0, seed=42)            # warm-up run
            r = p.cpals(max_iters=it, tol=0.0, seed=42)
            res[prec] = r
            # plain sweeps launched from the host (every mode gathers in this
            # precision): one untimed, then args.bf16_sweeps timed
            if args.bf16_sweeps > 0:
                p.sweep()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(args.bf16_sweeps):
                    p.sweep()
                e1.record(stream)
                e1.synchronize()
                sweep_ms[prec] = e0.elapsed_time(e1) / args.bf16_sweeps
            p.close()
            torch.cuda.synchronize()
        f32, b16 = res["fp32"], res["bf16"]
        ips = {k: v["iters_done"] / v["total_time_s"] for k, v in res.items()}
        out[layout] = {"fp32_iter_per_s": ips["fp32"], "bf16_iter_per_s": ips["bf16"],
                       "bf16_speedup": ips["bf16"] / ips["fp32"],
                       "fp32_sweep_ms": sweep_ms.get("fp32"), "bf16_sweep_ms": sweep_ms.get("bf16"),
                       "fp32_final_fit": f32["final_fit"], "bf16_final_fit": b16["final_fit"],
                       "max_abs_fit_diff_bf16_vs_fp32": float(np.max(np.abs(
                           b16["fit_history"] - f32["fit_history"])))}
    return out


def batched_block(device, stream, args):
    """The two batched CP-ALS workloads, each against the same runs one by
    one (Gauss-Seidel, FP64 solve, NCopy layout; the second call of each is
    timed, after a first call on the same plans):
      * 16 random restarts of rank 16 on 400,000 x 300,000 x 2,000 from 50M
        Zipf(1.0) draws, rank-8 |N(0,1)| truth + 2% noise: one plan of rank
        256 (dgpu_cpals_multistart) vs 16 plans of rank 16, 10 iterations;
      * 32 tensors, dims log-uniform in [1e3, 1e5], nnz log-uniform in
        [1e4, 5e6], rank-4 truth + 1% noise, rank 8, 30 iterations, tol 1e-4:
        dgpu_cpals_batch vs dgpu_cpals per tensor."""
    import torch
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    out = {}
    dims, vals, idx = synth.cp_zipf_torch((400_000, 300_000, 2_000), 50_000_000, (1.0, 1.0, 1.0),
                                          8, 0.02, 4, "cuda")
    K, Re, it = 16, 16, 10
    p = d.Plan(dims, vals, idx, threads=args.threads, rank=K * Re, layout="ncopy", device=device)
    p.set_stream(stream)
    p.cpals_multistart(K, max_iters=it, tol=0.0, seed=42)
    t0 = time.time()
    p.cpals_multistart(K, max_iters=it, tol=0.0, seed=42)
    tb = time.time() - t0
    p.close()
    single = []
    for k in range(K):
        q = d.Plan(dims, vals, idx, threads=args.threads, rank=Re, layout="ncopy", device=device)
        q.set_stream(stream)
        q.cpals(max_iters=it, tol=0.0, seed=42 + k)
        t0 = time.time()
        q.cpals(max_iters=it, tol=0.0, seed=42 + k)
        single.append(time.time() - t0)
        q.close()
    out["restarts"] = {"workload": f"400000x300000x2000, {len(vals)} nnz, {K} restarts x rank {Re}, "
                                   f"{it} iterations", "batched_s": tb, "one_by_one_s": sum(single),
                       "speedup": sum(single) / tb}
    del dims, vals, idx
    ts = synth.tensor_batch(32, seed=17)
    plans = [d.Plan(dm, v, i, threads=args.threads, rank=8, layout="ncopy", device=device)
             for dm, v, i in ts]
    t0 = time.time()
    d.cpals_batch(plans, max_iters=30, tol=1e-4, seed=42)
    cold = time.time() - t0
    t0 = time.time()
    d.cpals_batch(plans, max_iters=30, tol=1e-4, seed=42)
    tb = time.time() - t0
    one, one_cold = 0.0, 0.0
    for pl in plans:
        t0 = time.time()
        pl.cpals(max_iters=30, tol=1e-4, seed=42)
        one_cold += time.time() - t0
        t0 = time.time()
        pl.cpals(max_iters=30, tol=1e-4, seed=42)
        one += time.time() - t0
    for pl in plans:
        pl.close()
    out["tensors"] = {"workload": f"32 tensors, {sum(len(v) for _, v, _ in ts)} nnz in all, rank 8, "
                                  "30 iterations, tol 1e-4",
                      "batched_s": tb, "one_by_one_s": one, "speedup": one / tb,
                      "first_call_batched_s": cold, "first_call_one_by_one_s": one_cold}
    torch.cuda.synchronize()
    return out


def cpopt_block(device, stream, args):
    """CP-OPT forward (model values at the nonzeros, FP32, to a host buffer)
    and gradient (every factor's, to host buffers) on 100,000 x 100,000 x
    1,000 with 20M uniform nonzeros, N(0,1) values, rank 32, factors
    N(0, 0.1); NCopy and PingPong plans; 3 timed calls after one warm-up,
    into the host buffers the warm-up call allocated."""
    import torch
    import dynasor_plus_b200 as d
    from dynasor_plus_b200 import synth
    dims, vals, idx = synth.uniform((100_000, 100_000, 1_000), 20_000_000, seed=21, values="normal")
    rng = np.random.default_rng(22)
    Y = [np.asarray(rng.normal(0, 0.1, (int(n), 32)), np.float32) for n in dims]
    out = {"workload": "100000x100000x1000, 20M uniform nnz, rank 32", "nnz": len(vals)}
    for layout in ("ncopy", "pingpong"):
        p = d.Plan(dims, vals, idx, threads=args.threads, rank=32, layout=layout, device=device)
        p.set_stream(stream)
        for n in range(3):
            p.set_factor(n, Y[n])
        # the host buffers are allocated (and first touched) by the warm-up
        # calls and reused by the timed ones
        mv = p.model_values()
        gr = p.cpopt_gradient()
        torch.cuda.synchronize()
        t0 = time.time()
        for _ in range(3):
            p.model_values(out=mv)
        tf = (time.time() - t0) / 3
        t0 = time.time()
        for _ in range(3):
            p.cpopt_gradient(out=gr)
        tg = (time.time() - t0) / 3
        out[layout] = {"forward_ms": tf * 1e3, "forward_gnnz_s": len(vals) / tf / 1e9,
                       "gradient_ms": tg * 1e3, "gradient_gnnz_s": len(vals) / tg / 1e9}
        p.close()
    return out


def uniform_factors(dims, R, seed=42):
    rng = np.random.default_rng(seed)
    Rp = (R + 15) // 16 * 16
    Y = []
    for d in dims:
        y = np.zeros((int(d), Rp), np.float32)
        y[:, :R] = rng.random((int(d), R), dtype=np.float32)
        Y.append(y)
    return Y


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------------------
#  reference arm / CPU baseline
# ---------------------------------------------------------------------------
def reference_sweeps(dims, vals, idx, threads, R, warmup, steps, fiber_off=False, layout="pingpong"):
    from oracle import bindings as B
    ref = B.Reference(dims, vals, idx)
    ref.build(threads, layout)
    ref.factors(R)
    Y = uniform_factors(dims, R)
    for n in range(len(dims)):
        ref.set_Y(n, Y[n])
    ref.sweep_begin(fiber_off=fiber_off)
    times = []
    for s in range(warmup + steps):
        t = 0.0
        for n in range(len(dims)):
            t += ref.process(n)
        if s >= warmup:
            times.append(t)
    return times


def max_over_ranks(x: float, ws: int, device="cuda") -> float:
    """The largest of every rank's x (the job's time is its slowest rank)."""
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gnnz_s(nnz_per_rank: int, ws: int, ms_step: float) -> float:
    """Whole-job throughput of ws replicas, each sweeping nnz_per_rank
    nonzeros per step, timed by the slowest rank's ms per step."""
    return ws * nnz_per_rank / (ms_step * 1e-3) / 1e9


def run_reference_arm(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    from oracle import bindings as B
    if not B.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref was not built (the reference tree was absent at build time)"}))
        return
    try:
        dims, vals, idx = make_workload(args, "cuda")
    except Exception:
        dims, vals, idx = make_workload(args, "cpu")
    cores = os.cpu_count() or 1
    # every step is one reference sweep of the whole tensor (~2-5 s on 16
    # host cores), so W + K sweeps of the default run take a few minutes
    times = reference_sweeps(dims, vals, idx, cores, args.rank, args.warmup, args.steps)
    t = statistics.median(times)
    nnz = len(vals)
    val = nnz / t / 1e9
    out = {
        "metric": METRIC, "value": val, "unit": "GNNZ/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": f"zipf{ZIPF_S} 3-mode {DIMS[0]}x{DIMS[1]}x{DIMS[2]}, {args.draws} "
                               f"draws deduped to {nnz} nnz, rank {args.rank}",
                   "nnz": nnz, "layout": "pingpong", "threads": cores,
                   "fiber": "reference default", "timing": "median sweep"},
        "cpu_baseline": {"value": val, "unit": "GNNZ/s", "cores": cores, "kind": "reference",
                         "sample": f"the whole tensor ({nnz} nonzeros), one sweep per step, "
                                   f"PingPong layout, --threads {cores}"},
        "e2e": {"value": val, "unit": "GNNZ/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        # the reference's fastest layout (NCopy: no remap) on the same tensor
        tn = statistics.median(reference_sweeps(dims, vals, idx, cores, args.rank, 1, 3,
                                                layout="ncopy"))
        out["ncopy"] = {"value": nnz / tn / 1e9, "unit": "GNNZ/s", "ms_per_step": tn * 1e3}
    except Exception as ex:  # reported, never required
        out["ncopy"] = {"error": str(ex)[:200]}
    try:
        out["cpals_small"] = {"workload": "200x200x200, 100k nnz, rank 16, GS, tol 1e-4",
                              "threads": cores, **cpals_small_reference(cores)}
    except Exception as ex:  # reported, never required
        out["cpals_small"] = {"error": str(ex)[:200]}
    print(json.dumps(out))


# ---------------------------------------------------------------------------
#  B200 arm
# ---------------------------------------------------------------------------
def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    import torch
    import dynasor_plus_b200 as d

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    dims, vals, idx = make_workload(args, "cuda")
    nnz = len(vals)
    N = len(dims)
    t0 = time.time()
    plan = d.Plan(dims, vals, idx, threads=args.threads, rank=args.rank, layout=args.layout,
                  fiber=bool(args.fiber), precision=args.precision, device=local)
    build_s = time.time() - t0
    layout_used = plan.info()["layout"]
    stream = torch.cuda.Stream(device=local)
    plan.set_stream(stream)
    Y = uniform_factors(dims, args.rank)
    for n in range(N):
        plan.set_factor(n, Y[n])

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    # warm-up
    for _ in range(args.warmup):
        plan.sweep()
    plan.sync()

    clk = ClockSampler(local)
    clk.start()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clk.begin()
    e0.record(stream)
    for _ in range(args.steps):
        plan.sweep()
    e1.record(stream)
    e1.synchronize()
    clk.end()
    torch.cuda.synchronize()
    barrier()
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), ws)
    ms_step = ms / args.steps
    value = job_gnnz_s(nnz, ws, ms_step)

    # per-kernel timing pass (outside the timed region)
    plan.set_timing(True)
    plan.timing(reset=True)
    for _ in range(2):
        plan.sweep()
    tim = plan.timing(reset=True)
    plan.set_timing(False)
    launches_per_step = sum(v["launches"] for v in tim.values()) // 2

    # e2e through the host API with pinned buffers
    Rp = plan.Rp
    Yp = [torch.from_numpy(y).pin_memory() for y in Y]
    Op = [torch.empty((int(dims[n]), Rp), dtype=torch.float32).pin_memory() for n in range(N)]
    import ctypes as C
    Yptr = (C.c_void_p * N)(*[t.data_ptr() for t in Yp])
    Optr = (C.c_void_p * N)(*[t.data_ptr() for t in Op])
    L = d.lib()
    secs = C.c_double(0)
    for _ in range(max(1, args.warmup)):
        d.check(L.dgpu_mttkrp_sweep_host(plan._h, Yptr, Optr, C.byref(secs)))
    barrier()
    torch.cuda.synchronize()
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(args.steps):
        d.check(L.dgpu_mttkrp_sweep_host(plan._h, Yptr, Optr, C.byref(secs)))
    a1.record(stream)
    a1.synchronize()
    e2e_ms = max_over_ranks(a0.elapsed_time(a1) / args.steps, ws)
    fbytes = sum(int(dims[n]) * Rp * 4 for n in range(N))

    # roofline of the dominant kernel (largest device-time share)
    peak, peak_src = peaks()
    dom = max(tim, key=lambda k: tim[k]["total_ms"])
    dk = tim[dom]
    dom_ms = dk["total_ms"] / max(1, dk["launches"])
    dom_bytes = dk["bytes"] / max(1, dk["launches"])
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    total_ms = sum(v["total_ms"] for v in tim.values())
    sweep_bytes = sum(v["bytes"] for v in tim.values()) / 2
    # the algorithmic bytes of a sweep with remap: per mode the
    # slab read + the remap write + other factors once + Yhat once
    R = args.rank
    algo = 0.0
    for n in range(N):
        algo += 2 * nnz * (4 + 4 * N) + int(dims[n]) * R * 4
        algo += sum(int(dims[w]) * R * (2 if args.precision == "bf16" else 4) for w in range(N) if w != n)

    out = {
        "metric": METRIC, "value": value, "unit": "GNNZ/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "bf16-gather/f32-acc",
        "data": "synthetic",
        "config": {"workload": f"zipf{ZIPF_S} 3-mode {DIMS[0]}x{DIMS[1]}x{DIMS[2]}, {args.draws} draws "
                               f"deduped to {nnz} nnz, rank {args.rank}",
                   "nnz": nnz, "layout": layout_used, "threads": args.threads,
                   "fiber": bool(args.fiber), "precision": args.precision,
                   "l2": "inputs larger than L2 (slab %.2f GB)" % (nnz * (4 + 4 * N) / 1e9),
                   "parallelism": f"replicas x{ws}", "plan_build_s": round(build_s, 3)},
        "per_mode_gnnz_s": ws * nnz * N / (ms_step * 1e-3) / 1e9,
        "sweep_roofline": {"algorithmic_bytes": algo, "achieved_gbs": algo / (ms_step * 1e-3) / 1e9,
                           "peak_gbs": peak, "frac": algo / (ms_step * 1e-3) / 1e9 / peak,
                           "peak_source": peak_src},
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (NCU_DRAM_BYTES_PER_LAUNCH[dom] * nnz / NCU_NNZ
                                 if dom in NCU_DRAM_BYTES_PER_LAUNCH else None),
                     "traffic_source": ("ncu dram bytes per launch at this size" if nnz == NCU_NNZ
                                        else "ncu dram bytes per launch at 64,659,576 nnz, "
                                             "scaled by nnz"),
                     "peak_source": peak_src, "avg_launch_ms": dom_ms,
                     "algorithmic_bytes_per_launch": dom_bytes},
        "kernel_rooflines": {
            k: {"achieved_gbs": (v["bytes"] / v["launches"]) / (v["total_ms"] / v["launches"] * 1e-3) / 1e9,
                "frac": (v["bytes"] / v["launches"]) / (v["total_ms"] / v["launches"] * 1e-3) / 1e9 / peak,
                "avg_launch_ms": v["total_ms"] / v["launches"],
                "algorithmic_bytes_per_launch": v["bytes"] / v["launches"],
                "traffic_per_launch": (NCU_DRAM_BYTES_PER_LAUNCH[k] * nnz / NCU_NNZ
                                       if k in NCU_DRAM_BYTES_PER_LAUNCH else None)}
            for k, v in tim.items() if v["launches"] and v["total_ms"] > 0},
        "kernel_times_ms_per_step": {k: v["total_ms"] / 2 for k, v in tim.items() if v["launches"]},
        "kernel_share": {k: v["total_ms"] / total_ms for k, v in tim.items() if v["launches"]},
        "gpu_launches": launches_per_step * args.steps,
        "e2e": {"value": job_gnnz_s(nnz, ws, e2e_ms), "unit": "GNNZ/s",
                "h2d_bytes_per_step": fbytes, "d2h_bytes_per_step": fbytes,
                "ms_per_step": e2e_ms},
        "clocks": clocks,
    }

    # CP-ALS iterations/s on the same tensor (Gauss-Seidel, FP64 solve) and
    # on the small plain CP-ALS configuration
    if args.cpals_iters > 0:
        plan.cpals(max_iters=args.cpals_iters, tol=0.0, seed=42)     # warm-up run
        r = plan.cpals(max_iters=args.cpals_iters, tol=0.0, seed=42)
        out["cpals"] = {"iters": r["iters_done"], "iter_per_s": r["iters_done"] / r["total_time_s"],
                        "final_fit": r["final_fit"], "mttkrp_s": r["mttkrp_time_s"],
                        "linalg_s": r["linalg_time_s"]}
        if rank == 0:
            out["cpals_small"] = {"workload": "200x200x200, 100k nnz, rank 16, GS, tol 1e-4",
                                  "plan_threads": args.threads, **cpals_small_gpu(args.threads)}

    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            from oracle import bindings as B
            if B.ref_available():
                cores = os.cpu_count() or 1
                times = reference_sweeps(dims, vals, idx, cores, args.rank, 1, args.cpu_sweeps)
                t = statistics.median(times)
                out["cpu_baseline"] = {"value": nnz / t / 1e9, "unit": "GNNZ/s", "cores": cores,
                                       "kind": "reference",
                                       "sample": f"the whole tensor ({nnz} nonzeros): median of "
                                                 f"{args.cpu_sweeps} sweeps after one warm-up, "
                                                 f"PingPong layout, --threads {cores}"}
        except Exception as ex:  # the baseline is reported, never required
            out["cpu_baseline"] = {"value": None, "error": str(ex)[:200]}

    plan.close()

    # the same metric on the NCopy layout (one pre-sorted copy per mode, no
    # remap): the reference planner's choice when memory allows
    if rank == 0 and layout_used == "pingpong" and not args.no_ncopy:
        nc = d.Plan(dims, vals, idx, threads=args.threads, rank=args.rank, layout="ncopy",
                    fiber=bool(args.fiber), precision=args.precision, device=local)
        nc.set_stream(stream)
        for n in range(N):
            nc.set_factor(n, Y[n])
        for _ in range(args.warmup):
            nc.sweep()
        nc.sync()
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(args.steps):
            nc.sweep()
        c1.record(stream)
        c1.synchronize()
        nms = c0.elapsed_time(c1) / args.steps
        out["ncopy"] = {"value": nnz / (nms * 1e-3) / 1e9, "unit": "GNNZ/s", "ms_per_step": nms}
        if args.cpals_iters > 0:
            nc.cpals(max_iters=args.cpals_iters, tol=0.0, seed=42)       # warm-up run
            r = nc.cpals(max_iters=args.cpals_iters, tol=0.0, seed=42)
            out["ncopy"]["cpals"] = {"iters": r["iters_done"],
                                     "iter_per_s": r["iters_done"] / r["total_time_s"],
                                     "final_fit": r["final_fit"]}
        nc.close()
    if rank == 0 and not args.no_bf16 and args.cpals_iters > 0:
        try:
            out["bf16"] = bf16_block(local, stream, args)
        except Exception as ex:  # reported, never required
            out["bf16"] = {"error": str(ex)[:300]}
    if rank == 0 and not args.no_cpopt and args.cpals_iters > 0:
        try:
            out["cpopt"] = cpopt_block(local, stream, args)
        except Exception as ex:  # reported, never required
            out["cpopt"] = {"error": str(ex)[:300]}
    if rank == 0 and not args.no_batched and args.cpals_iters > 0:
        try:
            out["batched"] = batched_block(local, stream, args)
        except Exception as ex:  # reported, never required
            out["batched"] = {"error": str(ex)[:300]}
    if rank == 0:
        s = json.dumps(out)
        print(s)
        if args.json_out:
            with open(args.json_out, "w") as f:
                f.write(s + "\n")
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
