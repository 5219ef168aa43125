"""ctypes binding of libdynasor_b200.so (the C-ABI in include/dynasor_b200.h).

The library is loaded from this package directory only; there is no CPU
fallback.  ``lib()`` raises if the shared object is missing.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libdynasor_b200.so")
MAX_MODES = 8

OK = 0
ERRORS = {
    -1: "DGPU_ERR_ARG", -2: "DGPU_ERR_CUDA", -3: "DGPU_ERR_NOMEM", -4: "DGPU_ERR_EMPTY",
    -5: "DGPU_ERR_INDEX", -6: "DGPU_ERR_ORDER", -7: "DGPU_ERR_IO", -8: "DGPU_ERR_NOT_BUILT",
    -9: "DGPU_ERR_DEVICE",
}


class DgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class TensorDesc(C.Structure):
    _fields_ = [("num_modes", C.c_int), ("nnz", C.c_uint64),
                ("mode_size", C.POINTER(C.c_uint32)), ("vals", C.POINTER(C.c_float)),
                ("idx", C.POINTER(C.c_void_p))]


class PlanOpts(C.Structure):
    _fields_ = [("threads", C.c_int), ("rank", C.c_int), ("layout", C.c_int), ("fiber", C.c_int),
                ("precision", C.c_int), ("device", C.c_int), ("accum", C.c_int),
                ("mn_target", C.POINTER(C.c_uint32))]


class PlanInfo(C.Structure):
    _fields_ = [("num_modes", C.c_int), ("nnz", C.c_uint64), ("rank", C.c_int),
                ("rank_padded", C.c_int), ("threads", C.c_int),
                ("mode_size", C.c_uint32 * MAX_MODES), ("mn", C.c_uint32 * MAX_MODES),
                ("mn_shift", C.c_int * MAX_MODES), ("shards_per_mode", C.c_uint32 * MAX_MODES),
                ("kernel_class", C.c_int * MAX_MODES), ("avg_fiber_len", C.c_double * MAX_MODES),
                ("tiles", C.c_uint32 * MAX_MODES), ("next_mode", C.c_int),
                ("device_bytes", C.c_uint64), ("layout", C.c_int)]


class DnpInfo(C.Structure):
    _fields_ = [("layout_kind", C.c_int), ("num_modes", C.c_int), ("nnz", C.c_uint64),
                ("mode_size", C.c_uint32 * MAX_MODES), ("num_threads", C.c_int)]


class CpOptions(C.Structure):
    _fields_ = [("max_iters", C.c_int), ("tol", C.c_double), ("seed", C.c_uint64),
                ("ridge", C.c_double), ("kernel", C.c_int), ("solve_fp64", C.c_int),
                ("use_init", C.c_int), ("verbose", C.c_int), ("graphs", C.c_int)]


class CpResult(C.Structure):
    _fields_ = [("iters_done", C.c_int), ("final_fit", C.c_double), ("final_residual", C.c_double),
                ("tensor_norm", C.c_double), ("total_time_s", C.c_double),
                ("mttkrp_time_s", C.c_double), ("linalg_time_s", C.c_double)]


class ComputePlanInput(C.Structure):
    _fields_ = [("num_modes", C.c_int), ("nnz", C.c_uint64), ("mode_size", C.c_uint32 * MAX_MODES),
                ("rank_padded", C.c_int), ("threads", C.c_int), ("layout", C.c_int),
                ("fiber", C.c_int), ("kernel_class", C.c_int * MAX_MODES),
                ("avg_fiber_len", C.c_double * MAX_MODES), ("host_avail_bytes", C.c_uint64)]


class ComputePlan(C.Structure):
    _fields_ = [("layout", C.c_int), ("kernel", C.c_int), ("kernel_reason", C.c_char * 48),
                ("kernel_source", C.c_char * 16), ("per_mode", C.c_int * MAX_MODES),
                ("accum", C.c_int * MAX_MODES), ("rank_tile", C.c_int * MAX_MODES),
                ("precision", C.c_int), ("num_modes", C.c_int), ("rank_padded", C.c_int),
                ("threads", C.c_int), ("ofibs_bytes", C.c_uint64), ("factor_bytes", C.c_uint64),
                ("budget_bytes", C.c_uint64), ("device_bytes", C.c_uint64)]


class TuneResult(C.Structure):
    _fields_ = [("fiber_digit_bits", C.c_int), ("sort_digit_bits", C.c_int),
                ("chunks_per_sm", C.c_int), ("seg_chunk_tiles", C.c_int),
                ("mttkrp_ctas_per_sm", C.c_int), ("mttkrp_gather", C.c_int),
                ("candidates", C.c_int),
                ("default_ms", C.c_double), ("tuned_ms", C.c_double)]


class KernelTiming(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("launches", C.c_uint64), ("total_ms", C.c_double),
                ("bytes", C.c_double)]


class Coo(C.Structure):
    _fields_ = [("num_modes", C.c_int), ("nnz", C.c_uint64), ("mode_size", C.c_uint32 * MAX_MODES),
                ("vals", C.POINTER(C.c_float)), ("idx", C.c_void_p * MAX_MODES)]


# name -> (restype, argtypes)
_SIGS = {
    "dgpu_last_error": (C.c_char_p, []),
    "dgpu_version": (C.c_int, []),
    "dgpu_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "dgpu_plan_opts_default": (None, [C.POINTER(PlanOpts)]),
    "dgpu_plan_create": (C.c_int, [C.POINTER(TensorDesc), C.POINTER(PlanOpts), C.POINTER(C.c_void_p)]),
    "dgpu_plan_destroy": (C.c_int, [C.c_void_p]),
    "dgpu_dnp_peek": (C.c_int, [C.c_char_p, C.POINTER(DnpInfo)]),
    "dgpu_plan_create_from_dnp": (C.c_int, [C.c_char_p, C.POINTER(PlanOpts), C.POINTER(C.c_void_p)]),
    "dgpu_plan_save_dnp": (C.c_int, [C.c_void_p, C.c_char_p]),
    "dgpu_plan_morton": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dgpu_plan_get_info": (C.c_int, [C.c_void_p, C.POINTER(PlanInfo)]),
    "dgpu_plan_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "dgpu_plan_sync": (C.c_int, [C.c_void_p]),
    "dgpu_plan_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "dgpu_plan_get_timing": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_int]),
    "dgpu_plan_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(TuneResult)]),
    "dgpu_plan_shards": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "dgpu_plan_schedule": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                     C.POINTER(C.c_uint32)]),
    "dgpu_upload_factor": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "dgpu_download_factor": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "dgpu_download_yhat": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "dgpu_download_lambda": (C.c_int, [C.c_void_p, C.c_void_p]),
    "dgpu_factor_device_ptr": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p),
                                         C.POINTER(C.c_void_p)]),
    "dgpu_mttkrp_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "dgpu_mttkrp_sweep": (C.c_int, [C.c_void_p]),
    "dgpu_mttkrp_all_modes": (C.c_int, [C.c_void_p]),
    "dgpu_mttkrp_sweep_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]),
    "dgpu_download_slab": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "dgpu_download_copy": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "dgpu_cp_options_default": (None, [C.POINTER(CpOptions)]),
    "dgpu_cpals": (C.c_int, [C.c_void_p, C.POINTER(CpOptions), C.POINTER(CpResult), C.c_void_p]),
    "dgpu_init_factor": (C.c_int, [C.c_uint64, C.c_int, C.c_uint32, C.c_int, C.c_int, C.c_void_p]),
    "dgpu_cpals_multistart": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(CpOptions), C.c_void_p,
                                        C.c_void_p]),
    "dgpu_cpals_batch": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(CpOptions), C.c_void_p,
                                   C.c_void_p]),
    "dgpu_compute_plan_decide": (C.c_int, [C.POINTER(ComputePlanInput), C.c_char_p,
                                           C.POINTER(ComputePlan)]),
    "dgpu_build_compute_plan": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(ComputePlan)]),
    "dgpu_format_compute_plan": (C.c_int, [C.POINTER(ComputePlan), C.c_char_p, C.c_char_p,
                                           C.c_size_t]),
    "dgpu_la_gram": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_void_p]),
    "dgpu_tensor_norm_sq": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "dgpu_model_values": (C.c_int, [C.c_void_p, C.c_void_p]),
    "dgpu_cpopt_gradient": (C.c_int, [C.c_void_p, C.c_void_p]),
    "dgpu_sort_slab_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_uint64, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_uint32]),
    "dgpu_load_coo_tensor": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(Coo)]),
    "dgpu_load_tns": (C.c_int, [C.c_char_p, C.POINTER(Coo)]),
    "dgpu_load_dnb": (C.c_int, [C.c_char_p, C.POINTER(Coo)]),
    "dgpu_save_dnb": (C.c_int, [C.c_char_p, C.POINTER(Coo)]),
    "dgpu_coo_free": (None, [C.POINTER(Coo)]),
    "dgpu_dump_factor_bin": (C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_int, C.c_int]),
}

_lib = None


def lib() -> C.CDLL:
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m dynasor_plus_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != OK:
        msg = lib().dgpu_last_error()
        raise DgpuError(rc, msg.decode() if msg else "")
