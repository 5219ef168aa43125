"""ctypes bindings for the CHECKERS (test infrastructure only).

* ``Oracle``    -- this project's CPU restatement (``oracle/liboracle.so``).
* ``Reference`` -- the unmodified reference sources compiled by
  ``oracle/Makefile`` into ``oracle/_ref/libdynref_{avx512,avx2}.so``.

Only ``tests/``, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module.  The product package never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def _ptr_array(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def cpu_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return " avx512f " in (line + " ")
    except OSError:
        pass
    return False


def ref_library_path() -> str:
    name = "libdynref_avx512.so" if cpu_has_avx512() else "libdynref_avx2.so"
    return os.path.join(REF_DIR, name)


def ref_available() -> bool:
    return os.path.exists(ref_library_path())


def oracle_available() -> bool:
    return os.path.exists(ORACLE_SO)


def padded_rank(R: int) -> int:
    """Row stride of a factor matrix: R rounded up to 16 floats (one 64 B
    line), as in src/dynasor_io.cpp:154-160."""
    return (R + 15) // 16 * 16


# ---------------------------------------------------------------------------
#  Oracle (CPU restatement)
# ---------------------------------------------------------------------------
_olib = None


def _oracle_lib():
    global _olib
    if _olib is None:
        L = C.CDLL(ORACLE_SO)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int, C.c_uint64, _u32p, _f32p, C.c_void_p, C.c_int]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_modes.argtypes = [C.c_void_p, _i32p, _u32p, _i32p]
        L.orc_shards.argtypes = [C.c_void_p, C.c_int, _u64p, _u64p]
        L.orc_schedule.restype = C.c_int
        L.orc_schedule.argtypes = [C.c_void_p, C.c_int, _u32p, _u32p]
        L.orc_cursors.restype = C.c_size_t
        L.orc_cursors.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_get_slab.argtypes = [C.c_void_p, _f32p, C.c_void_p]
        L.orc_set_slab.argtypes = [C.c_void_p, _f32p, C.c_void_p]
        L.orc_fiber_sort.argtypes = [C.c_void_p, C.c_int]
        L.orc_remap.argtypes = [C.c_void_p, C.c_int]
        L.orc_process_layout.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_ncopy.argtypes = [C.c_void_p, C.c_int, C.c_int, _f32p, C.c_void_p]
        L.orc_morton.restype = C.c_int
        L.orc_morton.argtypes = [C.c_int, C.c_uint64, _u32p, _f32p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_mttkrp_f32_fold.argtypes = [C.c_int, C.c_uint64, _f32p, C.c_void_p, C.c_int,
                                          C.c_int, C.c_void_p, _f32p, C.c_uint32]
        L.orc_mttkrp_f64.argtypes = [C.c_int, C.c_uint64, _f32p, C.c_void_p, C.c_int, C.c_int,
                                     C.c_int, C.c_void_p, _f64p, C.c_uint32]
        L.orc_model_values.argtypes = [C.c_int, C.c_uint64, C.c_void_p, C.c_int, C.c_int,
                                       C.c_void_p, C.c_void_p, _f64p]
        L.orc_init_factor.argtypes = [C.c_uint64, C.c_int, C.c_uint32, C.c_int, C.c_int, _f32p]
        L.orc_uniform_factors.argtypes = [C.c_uint64, C.c_int, _u32p, C.c_int, C.c_int, C.c_void_p]
        L.orc_cpals_f64.restype = C.c_int
        L.orc_cpals_f64.argtypes = [C.c_int, C.c_uint64, _u32p, _f32p, C.c_void_p, C.c_int,
                                    C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p,
                                    _f64p, _f64p, C.c_int]
        _olib = L
    return _olib


class Oracle:
    """FLYCOO plan + remap restated on the CPU for `threads` workers."""

    def __init__(self, dims, vals, idx, threads: int):
        self.L = _oracle_lib()
        self.N = len(dims)
        self.dims = np.ascontiguousarray(dims, np.uint32)
        self.nnz = int(len(vals))
        self.T = int(threads)
        vals = np.ascontiguousarray(vals, np.float32)
        idx = [np.ascontiguousarray(i, np.uint32) for i in idx]
        self.h = self.L.orc_create(self.N, self.nnz, self.dims, vals, _ptr_array(idx), self.T)
        self.shift = np.zeros(self.N, np.int32)
        self.K = np.zeros(self.N, np.uint32)
        self.kclass = np.zeros(self.N, np.int32)
        self.L.orc_modes(self.h, self.shift, self.K, self.kclass)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def shards(self, n):
        K = int(self.K[n])
        b = np.zeros(K, np.uint64)
        e = np.zeros(K, np.uint64)
        self.L.orc_shards(self.h, n, b, e)
        return b, e

    def schedule(self, n):
        counts = np.zeros(self.T, np.uint32)
        flat = np.zeros(int(self.K[n]), np.uint32)
        k = self.L.orc_schedule(self.h, n, counts, flat)
        return counts, flat[:k]

    def cursors(self, n):
        m = self.L.orc_cursors(self.h, n, None)
        out = np.zeros(m, np.uint64)
        self.L.orc_cursors(self.h, n, out.ctypes.data)
        return out

    def slab(self):
        v = np.zeros(self.nnz, np.float32)
        ix = [np.zeros(self.nnz, np.uint32) for _ in range(self.N)]
        self.L.orc_get_slab(self.h, v, _ptr_array(ix))
        return v, ix

    def set_slab(self, v, ix):
        ix = [np.ascontiguousarray(i, np.uint32) for i in ix]
        self.L.orc_set_slab(self.h, np.ascontiguousarray(v, np.float32), _ptr_array(ix))

    def fiber_sort(self, n):
        self.L.orc_fiber_sort(self.h, n)

    def remap(self, n):
        self.L.orc_remap(self.h, n)

    def process_layout(self, n, fiber_on=True):
        self.L.orc_process_layout(self.h, n, 1 if fiber_on else 0)

    def ncopy(self, k, fiber_on=True):
        v = np.zeros(self.nnz, np.float32)
        ix = [np.zeros(self.nnz, np.uint32) for _ in range(self.N)]
        self.L.orc_ncopy(self.h, k, 1 if fiber_on else 0, v, _ptr_array(ix))
        return v, ix


def mttkrp_f32_fold(vals, idx, n, Y, dim_n):
    """The reference kernel's FP32 arithmetic in the given slab order."""
    L = _oracle_lib()
    N = len(idx)
    Rp = Y[0].shape[1]
    out = np.zeros((dim_n, Rp), np.float32)
    idx = [np.ascontiguousarray(i, np.uint32) for i in idx]
    Y = [np.ascontiguousarray(y, np.float32) for y in Y]
    L.orc_mttkrp_f32_fold(N, len(vals), np.ascontiguousarray(vals, np.float32), _ptr_array(idx),
                          n, Rp, _ptr_array(Y), out, dim_n)
    return out


def morton(dims, vals, idx):
    """The oracle's Morton layout: (mask, bits, sorted keys, values), or None
    when the mode sizes need more than 64 key bits."""
    N = len(dims)
    mask = np.zeros(N, np.uint64)
    bits = np.zeros(N, np.uint8)
    keys = np.zeros(len(vals), np.uint64)
    vo = np.zeros(len(vals), np.float32)
    idx = [np.ascontiguousarray(i, np.uint32) for i in idx]
    rc = _oracle_lib().orc_morton(N, len(vals), np.ascontiguousarray(dims, np.uint32),
                                  np.ascontiguousarray(vals, np.float32), _ptr_array(idx),
                                  mask.ctypes.data, bits.ctypes.data, keys.ctypes.data,
                                  vo.ctypes.data)
    return None if rc != 0 else (mask, bits, keys, vo)


def mttkrp_f64(vals, idx, n, Y, R, dim_n):
    L = _oracle_lib()
    N = len(idx)
    Rp = Y[0].shape[1]
    out = np.zeros((dim_n, Rp), np.float64)
    idx = [np.ascontiguousarray(i, np.uint32) for i in idx]
    Y = [np.ascontiguousarray(y, np.float32) for y in Y]
    L.orc_mttkrp_f64(N, len(vals), np.ascontiguousarray(vals, np.float32), _ptr_array(idx),
                     n, R, Rp, _ptr_array(Y), out, dim_n)
    return out


def model_values(idx, Y, R, lam=None):
    L = _oracle_lib()
    N = len(idx)
    Rp = Y[0].shape[1]
    nnz = len(idx[0])
    out = np.zeros(nnz, np.float64)
    idx = [np.ascontiguousarray(i, np.uint32) for i in idx]
    Y = [np.ascontiguousarray(y, np.float32) for y in Y]
    lp = None
    if lam is not None:
        lam = np.ascontiguousarray(lam, np.float32)
        lp = lam.ctypes.data
    L.orc_model_values(N, nnz, _ptr_array(idx), R, Rp, _ptr_array(Y), lp, out)
    return out


def init_factor(seed, n, rows, R):
    Rp = padded_rank(R)
    Y = np.zeros((rows, Rp), np.float32)
    _oracle_lib().orc_init_factor(seed, n, rows, R, Rp, Y)
    return Y


def uniform_factors(seed, dims, R):
    Rp = padded_rank(R)
    Y = [np.zeros((int(d), Rp), np.float32) for d in dims]
    _oracle_lib().orc_uniform_factors(seed, len(dims), np.ascontiguousarray(dims, np.uint32),
                                      R, Rp, _ptr_array(Y))
    return Y


def cpals_f64(dims, vals, idx, R, max_iters, tol, seed=42, ridge=1e-10, Y0=None, jacobi=False,
              bf16_gathers=False, last_mode_fp32=False):
    """FP64 CP-ALS (Gauss-Seidel, or Jacobi: all MTTKRPs from the iteration's
    starting factors) from the reference's seed-`seed` N(0,1) init (or from
    Y0).  bf16_gathers: the MTTKRP reads factors rounded to BF16 (the
    arithmetic of the BF16-gather path, otherwise FP64).  Returns
    (fit_history, Y, lambda)."""
    L = _oracle_lib()
    N = len(dims)
    Rp = padded_rank(R)
    if Y0 is None:
        Y = [init_factor(seed, n, int(dims[n]), R) for n in range(N)]
    else:
        Y = [np.array(y, np.float32, copy=True) for y in Y0]
    fit = np.zeros(max_iters, np.float64)
    lam = np.zeros(R, np.float64)
    idx = [np.ascontiguousarray(i, np.uint32) for i in idx]
    it = L.orc_cpals_f64(N, len(vals), np.ascontiguousarray(dims, np.uint32),
                         np.ascontiguousarray(vals, np.float32), _ptr_array(idx), R, Rp,
                         max_iters, tol, ridge, _ptr_array(Y), fit, lam,
                         (1 if jacobi else 0) | (2 if bf16_gathers else 0)
                         | (4 if last_mode_fp32 else 0))
    return fit[:it], Y, lam


# ---------------------------------------------------------------------------
#  Reference (unmodified sources, compiled here)
# ---------------------------------------------------------------------------
_rlib = None


def _ref_lib():
    global _rlib
    if _rlib is None:
        L = C.CDLL(ref_library_path())
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_int, C.c_uint64, _u32p, _f32p, C.c_void_p, C.c_int]
        L.ref_destroy.argtypes = [C.c_void_p]
        L.ref_build_flycoo.restype = C.c_int
        L.ref_build_flycoo.argtypes = [C.c_void_p, C.c_int, C.c_char_p]
        L.ref_plan_modes.argtypes = [C.c_void_p, _i32p, _u32p, _i32p, _f64p]
        L.ref_plan_shards.argtypes = [C.c_void_p, C.c_int, _u64p, _u64p]
        L.ref_plan_schedule.restype = C.c_int
        L.ref_plan_schedule.argtypes = [C.c_void_p, C.c_int, _u32p, _u32p]
        L.ref_plan_cursors.restype = C.c_size_t
        L.ref_plan_cursors.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.ref_get_slab.argtypes = [C.c_void_p, _f32p, C.c_void_p]
        L.ref_get_ncopy.restype = C.c_int
        L.ref_get_ncopy.argtypes = [C.c_void_p, C.c_int, _f32p, C.c_void_p]
        L.ref_fiber_sort.argtypes = [C.c_void_p, C.c_int]
        L.ref_factors.restype = C.c_int
        L.ref_factors.argtypes = [C.c_void_p, C.c_int]
        L.ref_set_Y.argtypes = [C.c_void_p, C.c_int, _f32p]
        L.ref_get_Y.argtypes = [C.c_void_p, C.c_int, _f32p]
        L.ref_get_Yhat.argtypes = [C.c_void_p, C.c_int, _f32p]
        L.ref_sweep_begin.argtypes = [C.c_void_p, C.c_int]
        L.ref_sweep_process.restype = C.c_double
        L.ref_sweep_process.argtypes = [C.c_void_p, C.c_int]
        L.ref_reference_mttkrp.argtypes = [C.c_void_p]
        L.ref_cpals.restype = C.c_int
        L.ref_cpals.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_uint64, C.c_int, C.c_float,
                                C.c_int, _f64p, _f32p, C.c_void_p, C.c_void_p]
        L.ref_spmttkrp_dynasor.restype = C.c_double
        L.ref_spmttkrp_dynasor.argtypes = [C.c_void_p]
        L.ref_save_dnp.restype = C.c_int
        L.ref_save_dnp.argtypes = [C.c_void_p, C.c_char_p]
        L.ref_load_dnp.restype = C.c_void_p
        L.ref_load_dnp.argtypes = [C.c_char_p, C.c_int, C.c_int]
        L.ref_build_morton.restype = C.c_int
        L.ref_build_morton.argtypes = [C.c_void_p]
        L.ref_morton_get.restype = C.c_int
        L.ref_morton_get.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_compute_plan.restype = C.c_int
        L.ref_compute_plan.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_char_p, C.c_char_p,
                                       C.c_char_p, C.c_int, _i32p]
        L.ref_all_modes_morton.restype = C.c_double
        L.ref_all_modes_morton.argtypes = [C.c_void_p]
        _rlib = L
    return _rlib


class Reference:
    """The reference's Tensor + FactorMatrices driven through its own API."""

    LAYOUTS = {"pingpong": 0, "ncopy": 1, "inplace": 2}

    def __init__(self, dims, vals, idx, quiet=True):
        self.L = _ref_lib()
        self.N = len(dims)
        self.dims = np.ascontiguousarray(dims, np.uint32)
        self.nnz = int(len(vals))
        vals = np.ascontiguousarray(vals, np.float32)
        idx = [np.ascontiguousarray(i, np.uint32) for i in idx]
        self.h = self.L.ref_create(self.N, self.nnz, self.dims, vals, _ptr_array(idx),
                                   1 if quiet else 0)
        self.T = None
        self.Rp = None

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    @classmethod
    def from_dnp(cls, path, threads, quiet=True):
        """A tensor loaded by the reference's .dnp reader (load_dnp_tensor,
        src/dynasor_dnp.cpp:719-803); None when the reader rejects it."""
        import struct
        with open(path, "rb") as f:
            head = f.read(4 + 5 * 4 + 8 + 8 * 4)
        N, nnz = struct.unpack_from("<I", head, 20)[0], struct.unpack_from("<Q", head, 24)[0]
        dims = np.array(struct.unpack_from("<8I", head, 32)[:N], np.uint32)
        self = cls.__new__(cls)
        self.L = _ref_lib()
        self.h = self.L.ref_load_dnp(str(path).encode(), int(threads), 1 if quiet else 0)
        if not self.h:
            return None
        self.N, self.dims, self.nnz, self.Rp = N, dims, int(nnz), None
        self._plan_facts(threads)
        return self

    def build_morton(self):
        """build_morton_layout on the built tensor (src/dynasor_morton.cpp:143-352)."""
        assert self.L.ref_build_morton(self.h) == 0

    def morton(self):
        """(mask[N] u64, bits[N] u8, sorted keys u64, values f32)."""
        mask = np.zeros(self.N, np.uint64)
        bits = np.zeros(self.N, np.uint8)
        keys = np.zeros(self.nnz, np.uint64)
        vals = np.zeros(self.nnz, np.float32)
        rc = self.L.ref_morton_get(self.h, mask.ctypes.data, bits.ctypes.data, keys.ctypes.data,
                                   vals.ctypes.data)
        assert rc == 0
        return mask, bits, keys, vals

    def compute_plan(self, rank_padded, layout="pingpong", kernel_cli="auto"):
        """dyn_build_compute_plan on the built tensor: (kernel 0 GS / 1
        Jacobi, reason, per-mode kernel class list)."""
        reason = C.create_string_buffer(64)
        per = np.zeros(self.N, np.int32)
        k = self.L.ref_compute_plan(self.h, int(rank_padded), int(self.T), layout.encode(),
                                    kernel_cli.encode(), reason, 64, per)
        return k, reason.value.decode(), [int(x) for x in per]

    def all_modes_morton(self):
        return self.L.ref_all_modes_morton(self.h)

    def save_dnp(self, path):
        """save_dnp_tensor on the built tensor (src/dynasor_dnp.cpp:639-700)."""
        return self.L.ref_save_dnp(self.h, str(path).encode()) == 0

    def build(self, threads, layout="pingpong"):
        got = self.L.ref_build_flycoo(self.h, int(threads), layout.encode())
        assert got == self.LAYOUTS[layout], (got, layout)
        self._plan_facts(threads)

    def _plan_facts(self, threads):
        self.T = int(threads)
        self.shift = np.zeros(self.N, np.int32)
        self.K = np.zeros(self.N, np.uint32)
        self.kclass = np.zeros(self.N, np.int32)
        self.afl = np.zeros(self.N, np.float64)
        self.L.ref_plan_modes(self.h, self.shift, self.K, self.kclass, self.afl)

    def shards(self, n):
        K = int(self.K[n])
        b = np.zeros(K, np.uint64)
        e = np.zeros(K, np.uint64)
        self.L.ref_plan_shards(self.h, n, b, e)
        return b, e

    def schedule(self, n):
        counts = np.zeros(self.T, np.uint32)
        flat = np.zeros(int(self.K[n]), np.uint32)
        k = self.L.ref_plan_schedule(self.h, n, counts, flat)
        return counts, flat[:k]

    def cursors(self, n):
        m = self.L.ref_plan_cursors(self.h, n, None)
        out = np.zeros(m, np.uint64)
        self.L.ref_plan_cursors(self.h, n, out.ctypes.data)
        return out

    def slab(self):
        v = np.zeros(self.nnz, np.float32)
        ix = [np.zeros(self.nnz, np.uint32) for _ in range(self.N)]
        self.L.ref_get_slab(self.h, v, _ptr_array(ix))
        return v, ix

    def ncopy(self, k):
        v = np.zeros(self.nnz, np.float32)
        ix = [np.zeros(self.nnz, np.uint32) for _ in range(self.N)]
        rc = self.L.ref_get_ncopy(self.h, k, v, _ptr_array(ix))
        assert rc >= 0, rc
        return v, ix, bool(rc)

    def fiber_sort(self, n):
        self.L.ref_fiber_sort(self.h, n)

    def factors(self, R):
        self.Rp = self.L.ref_factors(self.h, R)
        return self.Rp

    def set_Y(self, n, Y):
        self.L.ref_set_Y(self.h, n, np.ascontiguousarray(Y, np.float32))

    def get_Y(self, n):
        out = np.zeros((int(self.dims[n]), self.Rp), np.float32)
        self.L.ref_get_Y(self.h, n, out)
        return out

    def yhat(self, n):
        out = np.zeros((int(self.dims[n]), self.Rp), np.float32)
        self.L.ref_get_Yhat(self.h, n, out)
        return out

    def sweep_begin(self, fiber_off=False):
        self.L.ref_sweep_begin(self.h, 1 if fiber_off else 0)

    def process(self, n):
        return self.L.ref_sweep_process(self.h, n)

    def reference_mttkrp(self):
        self.L.ref_reference_mttkrp(self.h)

    def spmttkrp_dynasor(self):
        return self.L.ref_spmttkrp_dynasor(self.h)

    def cpals(self, R, max_iters, tol, seed=42, kernel="gs", ridge=1e-10, fiber_off=False):
        if self.Rp is None:
            self.factors(R)
        fit = np.zeros(max_iters, np.float64)
        lam = np.zeros(R, np.float32)
        tot = C.c_double(0)
        mt = C.c_double(0)
        it = self.L.ref_cpals(self.h, max_iters, tol, seed, 1 if kernel == "jacobi" else 0,
                              ridge, 1 if fiber_off else 0, fit, lam, C.byref(tot), C.byref(mt))
        return fit[:it], lam, tot.value, mt.value
