"""dynasor_plus_b200 -- sparse MTTKRP / CP-ALS on the NVIDIA B200 (sm_100a).

Python mirror of the reference's host API for the MTTKRP / CP-ALS path, over
the C ABI of libdynasor_b200.so (include/dynasor_b200.h):

    reference (C++)                          here
    -----------------------------------      -----------------------------------
    build_flycoo(T, threads, ...)            Plan(dims, vals, idx, threads, rank)
    FactorMatrices::Y / Yhat                 Plan.set_factor / factor / yhat
    SpmttkrpSweep::process(n)                Plan.process(n)
    spmttkrp_dynasor(T, F, threads)          Plan.sweep() / spmttkrp_dynasor()
    spmttkrp_all_modes_dynasor(T, F, thr)    Plan.all_modes()
    cpals(T, F, CpOptions) -> CpResult       Plan.cpals(...) -> CpResult-like dict
    load_coo_tensor / save_dnb_tensor        load_coo_tensor / save_dnb_tensor

All compute runs in CUDA kernels of the library; nothing here computes on
the CPU, and every call raises DgpuError when the library reports a failure.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import (ComputePlan, ComputePlanInput, CpOptions, CpResult, Coo, DgpuError, DnpInfo,
                   PlanInfo, PlanOpts, TensorDesc, TuneResult, check, lib, LIB_PATH)

__all__ = ["Plan", "DgpuError", "cpals_batch", "padded_rank", "load_coo_tensor", "save_dnb_tensor",
           "dnp_peek",
           "spmttkrp_dynasor", "device_count", "LIB_PATH", "PINGPONG", "NCOPY", "MORTON", "AUTO"]

PINGPONG = 0
NCOPY = 1
MORTON = 4  # one sorted 64-bit interleaved key + value per nonzero (all-modes pass only)
AUTO = 16  # NCopy when its slabs fit the device-memory budget, else PingPong
LAYOUTS = {"pingpong": PINGPONG, "ncopy": NCOPY, "morton": MORTON, "auto": AUTO}
LAYOUT_NAMES = {PINGPONG: "pingpong", NCOPY: "ncopy", MORTON: "morton"}
PRECISIONS = {"fp32": 0, "bf16": 1}
ACCUMS = {"auto": 0, "rowrun": 1, "private": 2}


def _kernel_code(kernel) -> int:
    """CP-ALS kernel keyword -> DGPU_CP_* (the reference's --cp-kernel words)."""
    k = str(kernel).lower()
    if k in ("jacobi", "all-modes", "all_modes", "js"):
        return 1
    if k == "auto":
        return 2
    return 0


_IMPL = {0: "Element", 1: "Fiber", 2: "FiberCSR"}
_ACCUM = {0: "all-modes", 1: "rowrun", 2: "private"}
_LAYOUT = {0: "pingpong", 1: "ncopy", 4: "morton"}


def _compute_plan_dict(cp, N) -> dict:
    return {"layout": _LAYOUT.get(cp.layout, cp.layout),
            "kernel": "jacobi" if cp.kernel == 1 else "gs",
            "kernel_reason": cp.kernel_reason.decode(), "kernel_source": cp.kernel_source.decode(),
            "per_mode": [_IMPL[cp.per_mode[n]] for n in range(N)],
            "accum": [_ACCUM.get(cp.accum[n], cp.accum[n]) for n in range(N)],
            "rank_tile": list(cp.rank_tile[:N]),
            "precision": "bf16" if cp.precision == 1 else "fp32",
            "rank_padded": cp.rank_padded, "threads": cp.threads,
            "ofibs_bytes": int(cp.ofibs_bytes), "factor_bytes": int(cp.factor_bytes),
            "budget_bytes": int(cp.budget_bytes), "device_bytes": int(cp.device_bytes),
            "_raw": cp}


def compute_plan_decide(dims, nnz, rank, threads, layout="pingpong", fiber=True,
                        kernel_class=None, avg_fiber_len=None, host_avail_bytes=0,
                        kernel="auto") -> dict:
    """The compute plan's decisions from tensor facts alone (host only, no
    device): dyn_build_compute_plan's kernel rule and per-mode class
    (src/dynasor_preprocess.cpp:1179-1363)."""
    N = len(dims)
    inp = ComputePlanInput()
    inp.num_modes = N
    inp.nnz = int(nnz)
    for n in range(min(N, len(inp.mode_size))):    # more modes: rejected by the library
        inp.mode_size[n] = int(dims[n])
        inp.kernel_class[n] = int(kernel_class[n]) if kernel_class is not None else 0
        inp.avg_fiber_len[n] = float(avg_fiber_len[n]) if avg_fiber_len is not None else 0.0
    inp.rank_padded = padded_rank(rank)
    inp.threads = int(threads)
    inp.layout = {"pingpong": 0, "ncopy": 1, "morton": 4}[layout]
    inp.fiber = 1 if fiber else 0
    inp.host_avail_bytes = int(host_avail_bytes)
    cp = ComputePlan()
    check(lib().dgpu_compute_plan_decide(C.byref(inp), str(kernel).encode(), C.byref(cp)))
    return _compute_plan_dict(cp, N)


def format_compute_plan(plan_dict, prefix="[plan]") -> str:
    """The plan banner (dyn_print_compute_plan's rows)."""
    buf = C.create_string_buffer(2048)
    check(lib().dgpu_format_compute_plan(C.byref(plan_dict["_raw"]), prefix.encode(), buf, 2048))
    return buf.value.decode()


def padded_rank(R: int) -> int:
    """Row stride of a factor matrix: R rounded up to 16 floats (64 B), the
    reference's FactorMatrices::allocate padding (src/dynasor_io.cpp:154-160)."""
    return (int(R) + 15) // 16 * 16


def device_count() -> int:
    n = C.c_int(0)
    rc = lib().dgpu_device_count(C.byref(n))
    return n.value if rc == 0 else 0


def _ptrs(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


class Plan:
    """A FLYCOO tensor plan resident on one GPU (build_flycoo + FactorMatrices).

    dims   : mode sizes (I_0..I_{N-1})
    vals   : float32 [nnz]
    idx    : N uint32 arrays of 0-based indices
    threads: the reference worker count the plan is built for (--threads)
    rank   : R; factors are I_n x padded_rank(R) float32
    layout : "pingpong" (device remap every mode), "ncopy", "morton" (one
             sorted interleaved 64-bit key + value per nonzero; all-modes
             pass, sweeps and Jacobi CP-ALS only), or "auto" (NCopy
             when N+1 slabs fit 70% of free device memory less a headroom of
             max(2 GiB, 25% of total), else PingPong; info()["layout"] tells)
    fiber  : fiber-sort DenseFiber modes (reference default) or not
             (the reference's DYN_FIBER_OFF=1 layout)
    precision: "fp32" or "bf16" (BF16 factor gathers, FP32 accumulation)
    """

    def __init__(self, dims, vals, idx, threads: int, rank: int, layout: str = "pingpong",
                 fiber: bool = True, precision: str = "fp32", device: int = 0,
                 mn_target=None, stream=None, accum: str = "auto"):
        L = lib()
        self.N = len(dims)
        self.dims = np.ascontiguousarray(dims, np.uint32)
        self._vals = np.ascontiguousarray(vals, np.float32)
        self._idx = [np.ascontiguousarray(i, np.uint32) for i in idx]
        self.nnz = int(self._vals.shape[0])
        if len(self._idx) != self.N or any(i.shape[0] != self.nnz for i in self._idx):
            raise ValueError("idx must hold one array of nnz indices per mode")
        self.R = int(rank)
        self.Rp = padded_rank(rank)
        desc = TensorDesc(self.N, self.nnz, self.dims.ctypes.data_as(C.POINTER(C.c_uint32)),
                          self._vals.ctypes.data_as(C.POINTER(C.c_float)),
                          C.cast(_ptrs(self._idx), C.POINTER(C.c_void_p)))
        opts = PlanOpts()
        L.dgpu_plan_opts_default(C.byref(opts))
        opts.threads = int(threads)
        opts.rank = self.R
        opts.layout = LAYOUTS[layout]
        opts.fiber = 1 if fiber else 0
        opts.precision = PRECISIONS[precision]
        opts.device = int(device)
        opts.accum = ACCUMS[accum]
        self._mn = None
        if mn_target is not None:
            self._mn = np.ascontiguousarray(mn_target, np.uint32)
            opts.mn_target = self._mn.ctypes.data_as(C.POINTER(C.c_uint32))
        h = C.c_void_p()
        check(L.dgpu_plan_create(C.byref(desc), C.byref(opts), C.byref(h)))
        self._h = h
        # the plan keeps device copies; drop the host staging arrays
        self._vals = None
        self._idx = None
        if stream is not None:
            self.set_stream(stream)

    @classmethod
    def from_dnp(cls, path, threads: int, rank: int, precision: str = "fp32", device: int = 0,
                 stream=None, accum: str = "auto", fiber: bool = True) -> "Plan":
        """A plan from a .dnp processed-tensor file (the reference's
        runtime-only mode, load_dnp_tensor): its slab(s), shard tables and
        schedule are used as they are.  `threads` must equal the file's
        thread count; the file decides the layout (PingPong, NCopy or Morton).
        `fiber` applies to PingPong files (NCopy copies record it)."""
        L = lib()
        info = dnp_peek(path)
        self = cls.__new__(cls)
        self.N = info["num_modes"]
        self.dims = np.asarray(info["mode_size"], np.uint32)
        self.nnz = info["nnz"]
        self.R = int(rank)
        self.Rp = padded_rank(rank)
        self._vals = self._idx = self._mn = None
        opts = PlanOpts()
        L.dgpu_plan_opts_default(C.byref(opts))
        opts.threads = int(threads)
        opts.rank = self.R
        opts.fiber = 1 if fiber else 0
        opts.precision = PRECISIONS[precision]
        opts.device = int(device)
        opts.accum = ACCUMS[accum]
        h = C.c_void_p()
        check(L.dgpu_plan_create_from_dnp(os.fsencode(path), C.byref(opts), C.byref(h)))
        self._h = h
        if stream is not None:
            self.set_stream(stream)
        return self

    def morton(self, keys: bool = True):
        """Morton layout state: (mask[N] uint64, bits[N] uint8, sorted keys
        uint64[nnz], values float32[nnz]); keys/values None when keys=False."""
        mask = np.zeros(self.N, np.uint64)
        bits = np.zeros(self.N, np.uint8)
        k = np.zeros(self.nnz, np.uint64) if keys else None
        v = np.zeros(self.nnz, np.float32) if keys else None
        check(lib().dgpu_plan_morton(self._h, mask.ctypes.data, bits.ctypes.data,
                                     k.ctypes.data if keys else None,
                                     v.ctypes.data if keys else None))
        return mask, bits, k, v

    def save_dnp(self, path):
        """Write the plan as a .dnp file (save_dnp_tensor): PingPong plans
        between sweeps, NCopy plans any time."""
        check(lib().dgpu_plan_save_dnp(self._h, os.fsencode(path)))

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().dgpu_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- plan facts -----------------------------------------------------------
    def info(self) -> dict:
        inf = PlanInfo()
        check(lib().dgpu_plan_get_info(self._h, C.byref(inf)))
        N = inf.num_modes
        return {
            "num_modes": N, "nnz": inf.nnz, "rank": inf.rank, "rank_padded": inf.rank_padded,
            "threads": inf.threads, "mode_size": list(inf.mode_size[:N]), "mn": list(inf.mn[:N]),
            "mn_shift": list(inf.mn_shift[:N]), "shards_per_mode": list(inf.shards_per_mode[:N]),
            "kernel_class": list(inf.kernel_class[:N]),
            "avg_fiber_len": list(inf.avg_fiber_len[:N]), "tiles": list(inf.tiles[:N]),
            "next_mode": inf.next_mode, "device_bytes": inf.device_bytes,
            "layout": LAYOUT_NAMES.get(inf.layout, inf.layout),
        }

    def shards(self, n: int):
        K = self.info()["shards_per_mode"][n]
        b = np.zeros(K, np.uint64)
        e = np.zeros(K, np.uint64)
        check(lib().dgpu_plan_shards(self._h, n, b.ctypes.data, e.ctypes.data))
        return b, e

    def schedule(self, n: int):
        inf = self.info()
        counts = np.zeros(inf["threads"], np.uint32)
        flat = np.zeros(inf["shards_per_mode"][n], np.uint32)
        k = C.c_uint32(0)
        check(lib().dgpu_plan_schedule(self._h, n, counts.ctypes.data, flat.ctypes.data,
                                       C.byref(k)))
        return counts, flat[:k.value]

    def set_stream(self, stream):
        """Issue all device work on `stream` (an int handle or an object with
        a `cuda_stream` attribute, e.g. torch.cuda.Stream)."""
        handle = getattr(stream, "cuda_stream", stream)
        check(lib().dgpu_plan_set_stream(self._h, C.c_void_p(int(handle))))

    def sync(self):
        check(lib().dgpu_plan_sync(self._h))

    def set_timing(self, on: bool = True):
        """Bracket every kernel launch with CUDA events (see timing())."""
        check(lib().dgpu_plan_set_timing(self._h, 1 if on else 0))

    def timing(self, reset: bool = True) -> dict:
        """{kind: {"launches", "total_ms", "bytes"}} accumulated since the
        last reset (synchronises the plan stream)."""
        from ._lib import KernelTiming
        arr = (KernelTiming * 16)()
        n = C.c_int(0)
        check(lib().dgpu_plan_get_timing(self._h, arr, 16, C.byref(n), 1 if reset else 0))
        return {arr[i].name.decode(): {"launches": int(arr[i].launches),
                                       "total_ms": float(arr[i].total_ms),
                                       "bytes": float(arr[i].bytes)} for i in range(n.value)}

    # -- factors ---------------------------------------------------------------
    def set_factor(self, n: int, Y):
        Y = np.ascontiguousarray(Y, np.float32)
        if Y.shape != (int(self.dims[n]), self.Rp):
            raise ValueError(f"factor {n} must be {int(self.dims[n])} x {self.Rp}")
        check(lib().dgpu_upload_factor(self._h, n, Y.ctypes.data))
        self.sync()

    def factor(self, n: int):
        out = np.zeros((int(self.dims[n]), self.Rp), np.float32)
        check(lib().dgpu_download_factor(self._h, n, out.ctypes.data))
        return out

    def yhat(self, n: int):
        out = np.zeros((int(self.dims[n]), self.Rp), np.float32)
        check(lib().dgpu_download_yhat(self._h, n, out.ctypes.data))
        return out

    def lam(self):
        out = np.zeros(self.R, np.float32)
        check(lib().dgpu_download_lambda(self._h, out.ctypes.data))
        return out

    def device_ptrs(self, n: int):
        y, yh = C.c_void_p(), C.c_void_p()
        check(lib().dgpu_factor_device_ptr(self._h, n, C.byref(y), C.byref(yh)))
        return y.value, yh.value

    # -- MTTKRP -------------------------------------------------------------------
    def process(self, n: int):
        """SpmttkrpSweep::process(n): Yhat[n] and (PingPong) the device remap."""
        check(lib().dgpu_mttkrp_mode(self._h, int(n)))

    def sweep(self):
        check(lib().dgpu_mttkrp_sweep(self._h))

    def all_modes(self):
        check(lib().dgpu_mttkrp_all_modes(self._h))

    def sweep_host(self, Y):
        """Upload Y[0..N-1] (host), one sweep, download every Yhat; returns
        (list of Yhat, device seconds of the sweep)."""
        Y = [np.ascontiguousarray(y, np.float32) for y in Y]
        out = [np.zeros((int(self.dims[n]), self.Rp), np.float32) for n in range(self.N)]
        secs = C.c_double(0)
        check(lib().dgpu_mttkrp_sweep_host(self._h, _ptrs(Y), _ptrs(out), C.byref(secs)))
        return out, secs.value

    def slab(self):
        v = np.zeros(self.nnz, np.float32)
        ix = [np.zeros(self.nnz, np.uint32) for _ in range(self.N)]
        check(lib().dgpu_download_slab(self._h, v.ctypes.data, _ptrs(ix)))
        return v, ix

    def copy(self, k: int):
        v = np.zeros(self.nnz, np.float32)
        ix = [np.zeros(self.nnz, np.uint32) for _ in range(self.N)]
        check(lib().dgpu_download_copy(self._h, k, v.ctypes.data, _ptrs(ix)))
        return v, ix

    # -- CP-ALS / CP-OPT -------------------------------------------------------------
    def cpals(self, max_iters=50, tol=1e-4, seed=42, ridge=1e-10, kernel="gs",
              solve_fp64=True, use_init=False, verbose=False, graphs=True):
        o = CpOptions()
        lib().dgpu_cp_options_default(C.byref(o))
        o.max_iters = int(max_iters)
        o.tol = float(tol)
        o.seed = int(seed)
        o.ridge = float(ridge)
        o.kernel = _kernel_code(kernel)
        o.solve_fp64 = 1 if solve_fp64 else 0
        o.use_init = 1 if use_init else 0
        o.verbose = 1 if verbose else 0
        o.graphs = 1 if graphs else 0
        r = CpResult()
        hist = np.zeros(max(1, int(max_iters)), np.float64)
        check(lib().dgpu_cpals(self._h, C.byref(o), C.byref(r), hist.ctypes.data))
        return {
            "iters_done": r.iters_done, "final_fit": r.final_fit,
            "final_residual": r.final_residual, "tensor_norm": r.tensor_norm,
            "total_time_s": r.total_time_s, "mttkrp_time_s": r.mttkrp_time_s,
            "linalg_time_s": r.linalg_time_s, "fit_history": hist[:r.iters_done].copy(),
            "lambda": self.lam(),
        }

    def cpals_multistart(self, restarts, max_iters=50, tol=1e-4, seed=42, ridge=1e-10,
                         kernel="gs", solve_fp64=True, use_init=False, verbose=False, graphs=True):
        """`restarts` CP-ALS runs in this plan (rank = restarts x per-restart
        rank); restart k starts from seed + k.  Returns one result dict per
        restart; its factor columns are [k*Re, (k+1)*Re) of every factor."""
        o = CpOptions()
        lib().dgpu_cp_options_default(C.byref(o))
        o.max_iters = int(max_iters)
        o.tol = float(tol)
        o.seed = int(seed)
        o.ridge = float(ridge)
        o.kernel = _kernel_code(kernel)
        o.solve_fp64 = 1 if solve_fp64 else 0
        o.use_init = 1 if use_init else 0
        o.verbose = 1 if verbose else 0
        o.graphs = 1 if graphs else 0
        K = int(restarts)
        res = (CpResult * K)()
        hist = np.zeros((K, max(1, int(max_iters))), np.float64)
        check(lib().dgpu_cpals_multistart(self._h, K, C.byref(o), C.cast(res, C.c_void_p),
                                          hist.ctypes.data))
        lam = self.lam()
        Re = self.R // K
        return [{"iters_done": r.iters_done, "final_fit": r.final_fit,
                 "final_residual": r.final_residual, "tensor_norm": r.tensor_norm,
                 "total_time_s": r.total_time_s,
                 "fit_history": hist[k, :r.iters_done].copy(),
                 "lambda": lam[k * Re:(k + 1) * Re].copy()} for k, r in enumerate(res)]

    def autotune(self, sweeps: int = 2) -> dict:
        """dgpu_plan_autotune: partition chunk sizes, digit widths and the
        MTTKRP grid target chosen by timing whole sweeps (the slab advances
        by the sweeps timed; no permutation depends on the knobs)."""
        r = TuneResult()
        check(lib().dgpu_plan_autotune(self._h, int(sweeps), C.byref(r)))
        return {k: getattr(r, k) for k, _ in TuneResult._fields_}

    def compute_plan(self, kernel="auto") -> dict:
        """dyn_build_compute_plan for this plan: the CP-ALS kernel the
        reference's rule picks, the per-mode kernel class, and what this
        engine runs per mode (accumulation scheme, rank tile)."""
        cp = ComputePlan()
        check(lib().dgpu_build_compute_plan(self._h, str(kernel).encode(), C.byref(cp)))
        return _compute_plan_dict(cp, self.N)

    def tensor_norm_sq(self) -> float:
        out = C.c_double(0)
        check(lib().dgpu_tensor_norm_sq(self._h, C.byref(out)))
        return out.value

    def model_values(self, out=None):
        """CP model at every nonzero of the current slab (FP32).  `out`: a
        C-contiguous float32 array of nnz entries to write into (reused
        across calls, it saves allocating and first touching the pages)."""
        if out is None:
            out = np.empty(self.nnz, np.float32)
        elif out.dtype != np.float32 or out.size != self.nnz or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of nnz entries")
        check(lib().dgpu_model_values(self._h, out.ctypes.data))
        return out

    def cpopt_gradient(self, out=None):
        """d(0.5*||X - M||^2)/dY[n] for every n (list of I_n x Rp float32).
        `out`: such a list to write into (reused across calls)."""
        if out is None:
            out = [np.empty((int(self.dims[n]), self.Rp), np.float32) for n in range(self.N)]
        else:
            for n, o in enumerate(out):
                if (o.dtype != np.float32 or o.shape != (int(self.dims[n]), self.Rp)
                        or not o.flags.c_contiguous):
                    raise ValueError(f"out[{n}] must be a C-contiguous float32 I_n x Rp array")
        check(lib().dgpu_cpopt_gradient(self._h, _ptrs(out)))
        return out


def init_factor(seed: int, n: int, rows: int, rank: int):
    """The reference's seeded N(0,1) initial factor of mode n (host only):
    rows x Rp float32, padding zero -- what cpals starts from."""
    Rp = padded_rank(rank)
    Y = np.zeros((int(rows), Rp), np.float32)
    check(lib().dgpu_init_factor(int(seed), int(n), int(rows), int(rank), Rp, Y.ctypes.data))
    return Y


def spmttkrp_dynasor(plan: Plan, Y):
    """One all-modes sweep from host factors; returns (Yhat list, seconds).
    Mirrors spmttkrp_dynasor (src/dynasor.cpp:545-559)."""
    return plan.sweep_host(Y)


# ---- loaders (host code inside the library) ----------------------------------
def _coo_to_numpy(c: Coo):
    N = c.num_modes
    nnz = int(c.nnz)
    dims = np.array(c.mode_size[:N], np.uint32)
    vals = np.ctypeslib.as_array(c.vals, shape=(nnz,)).copy() if nnz else np.zeros(0, np.float32)
    idx = []
    for n in range(N):
        p = C.cast(c.idx[n], C.POINTER(C.c_uint32))
        idx.append(np.ctypeslib.as_array(p, shape=(nnz,)).copy() if nnz else np.zeros(0, np.uint32))
    return dims, vals, idx


def load_coo_tensor(path: str, cache: bool = True):
    """load_coo_tensor (src/dynasor_io.cpp:1184-1261): `path`.dnb when it is
    fresh, else the .tns text (writing the .dnb cache when `cache`).
    Returns (dims, vals, idx) with 0-based indices."""
    c = Coo()
    check(lib().dgpu_load_coo_tensor(os.fsencode(path), 1 if cache else 0, C.byref(c)))
    try:
        return _coo_to_numpy(c)
    finally:
        lib().dgpu_coo_free(C.byref(c))


def load_dnb(path: str):
    c = Coo()
    check(lib().dgpu_load_dnb(os.fsencode(path), C.byref(c)))
    try:
        return _coo_to_numpy(c)
    finally:
        lib().dgpu_coo_free(C.byref(c))


DNP_LAYOUTS = {0: "morton", 1: "ncopy", 2: "pingpong", 3: "inplace"}


def dnp_peek(path) -> dict:
    """Header of a .dnp processed-tensor file (no device needed):
    layout, num_modes, nnz, mode_size and the thread count its schedule was
    built for (load_dnp_header / load_dnp_num_threads / load_dnp_layout)."""
    info = DnpInfo()
    check(lib().dgpu_dnp_peek(os.fsencode(path), C.byref(info)))
    N = info.num_modes
    return {"layout": DNP_LAYOUTS.get(info.layout_kind, info.layout_kind), "num_modes": N,
            "nnz": int(info.nnz), "mode_size": list(info.mode_size[:N]),
            "num_threads": info.num_threads}


def save_dnb_tensor(path: str, dims, vals, idx):
    """save_dnb_tensor (src/dynasor_io.cpp:854-893): DNB1 binary cache."""
    dims = np.ascontiguousarray(dims, np.uint32)
    vals = np.ascontiguousarray(vals, np.float32)
    idx = [np.ascontiguousarray(i, np.uint32) for i in idx]
    c = Coo()
    c.num_modes = len(dims)
    c.nnz = len(vals)
    for n in range(len(dims)):
        c.mode_size[n] = int(dims[n])
        c.idx[n] = idx[n].ctypes.data
    c.vals = vals.ctypes.data_as(C.POINTER(C.c_float))
    check(lib().dgpu_save_dnb(os.fsencode(path), C.byref(c)))


def dump_factor_matrix_bin(path: str, Y, R: int):
    """DYFM factor dump (src/dynasor_io.cpp:1287-1348)."""
    Y = np.ascontiguousarray(Y, np.float32)
    check(lib().dgpu_dump_factor_bin(os.fsencode(path), Y.ctypes.data, Y.shape[0], int(R), Y.shape[1]))


def cpals_batch(plans, max_iters=50, tol=1e-4, seed=42, ridge=1e-10, kernel="gs",
                solve_fp64=True, use_init=False, graphs=True):
    """Independent CP-ALS runs on several plans (one per tensor) whose
    iterations after the first run as parallel device loops of one graph
    launch.  Returns one result dict per plan (as Plan.cpals)."""
    o = CpOptions()
    lib().dgpu_cp_options_default(C.byref(o))
    o.max_iters = int(max_iters)
    o.tol = float(tol)
    o.seed = int(seed)
    o.ridge = float(ridge)
    o.kernel = _kernel_code(kernel)
    o.solve_fp64 = 1 if solve_fp64 else 0
    o.use_init = 1 if use_init else 0
    o.graphs = 1 if graphs else 0
    K = len(plans)
    hs = (C.c_void_p * K)(*[pl._h for pl in plans])
    res = (CpResult * K)()
    hist = np.zeros((K, max(1, int(max_iters))), np.float64)
    check(lib().dgpu_cpals_batch(C.cast(hs, C.c_void_p), K, C.byref(o), C.cast(res, C.c_void_p),
                                 hist.ctypes.data))
    return [{"iters_done": r.iters_done, "final_fit": r.final_fit,
             "final_residual": r.final_residual, "tensor_norm": r.tensor_norm,
             "total_time_s": r.total_time_s, "mttkrp_time_s": r.mttkrp_time_s,
             "linalg_time_s": r.linalg_time_s, "fit_history": hist[k, :r.iters_done].copy(),
             "lambda": plans[k].lam()} for k, r in enumerate(res)]

