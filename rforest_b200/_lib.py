"""Loader and ctypes signatures for libmpzmm_b200.so (include/mpzmm_b200.h)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmpzmm_b200.so")
CSRC = os.path.join(HERE, "csrc")

MPZMM_OK = 0
MPZMM_ERR_ARG = 1
MPZMM_ERR_TOO_LARGE = 2
MPZMM_ERR_CAPACITY = 3
MPZMM_ERR_CUDA = 4
MPZMM_ERR_NOMEM = 5
MPZMM_ERR_STATE = 6
MPZMM_ERR_TIMEOUT = 7
MPZMM_ERR_BUSY = 8
MPZMM_ERR_BOUNDS = 9

MPZMM_OPT_CONTRACT = 1
MPZMM_OPT_CHUNK_LIMBS = 2
MPZMM_OPT_CHECK_BOUNDS = 3
MPZMM_OPT_TEST_STALL_TC = 100
MPZMM_OPT_TEST_FAIL_ALLOC = 101
CONTRACT_AUTO, CONTRACT_CUDA_CORES, CONTRACT_TENSOR_CORES = 0, 1, 2

u64p = C.POINTER(C.c_uint64)
i64p = C.POINTER(C.c_int64)
i32p = C.POINTER(C.c_int32)


class Product(C.Structure):
    """struct mpzmm_product."""
    _fields_ = [
        ("m", C.c_int), ("k", C.c_int), ("n", C.c_int),
        ("a_limbs", u64p), ("a_offs", i64p), ("a_sizes", i32p),
        ("b_limbs", u64p), ("b_offs", i64p), ("b_sizes", i32p),
        ("c_limbs", u64p), ("c_offs", i64p), ("c_caps", i64p), ("c_sizes", i32p),
    ]


class Matrix(C.Structure):
    """struct mpzmm_matrix."""
    _fields_ = [
        ("rows", C.c_int), ("cols", C.c_int),
        ("limbs", u64p), ("offs", i64p), ("sizes", i32p),
    ]


class MpzmmError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"mpzmm status {status}: {message}")
        self.status = status


_lib = None


def build() -> None:
    """Compile the library in place (nvcc, sm_100a)."""
    subprocess.run(["make", "-s", "-C", CSRC, "-j8"], check=True)


def lib():
    """The loaded library.  Raises if the shared object is missing: there is no
    fallback implementation."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built (run __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "hw_mpz_setup": (None, []),
        "hw_mpz_clear": (None, []),
        "mpz_rmatrix_mult_fft": (None, [vp, vp, C.c_int, vp, C.c_int, vp]),
        "cu_mpz_rmatrix_mult_fft": (None, [vp, vp, C.c_int, vp, C.c_int, vp]),
        "mpz_rmatrix_gpu_fft_suitable": (C.c_int, [vp, C.c_int, vp, C.c_int]),
        "mpzmm_set_fatal_hook": (None, [vp]),
        "mpzmm_setup": (C.c_int, [C.c_int]),
        "mpzmm_set_option": (C.c_int, [C.c_int, C.c_int]),
        "mpzmm_get_option": (C.c_int, [C.c_int]),
        "mpzmm_autotune": (C.c_int, [vp, C.POINTER(C.c_float)]),
        "mpzmm_last_error": (C.c_char_p, []),
        "mpzmm_device_available": (C.c_int, []),
        "mpzmm_matmul": (C.c_int, [C.c_int, C.c_int, C.c_int, u64p, i64p, i32p, u64p, i64p,
                                   i32p, u64p, i64p, i64p, i32p, vp]),
        "mpzmm_output_limbs": (C.c_int64, [C.c_int, C.c_int64, C.c_int64]),
        "mpzmm_matmul_batch": (C.c_int, [C.c_int, C.POINTER(Product), vp]),
        "mpzmm_plan_create": (C.c_int, [C.POINTER(vp), C.c_int, C.POINTER(Product), vp]),
        "mpzmm_plan_execute": (C.c_int, [vp, vp]),
        "mpzmm_plan_download": (C.c_int, [vp, vp]),
        "mpzmm_plan_upload": (C.c_int, [vp, vp]),
        "mpzmm_plan_create_fixed_b": (C.c_int, [C.POINTER(vp), C.c_int, C.POINTER(Product), vp]),
        "mpzmm_plan_upload_a": (C.c_int, [vp, vp]),
        "mpzmm_plan_destroy": (None, [vp]),
        "mpzmm_plan_set_timing": (C.c_int, [vp, C.c_int]),
        "mpzmm_plan_set_graph": (C.c_int, [vp, C.c_int]),
        "mpzmm_plan_stage_times": (C.c_int, [vp, C.POINTER(C.c_float), i64p, i64p]),
        "mpzmm_plan_info": (C.c_int, [vp, i64p, i64p, C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "mpzmm_matmul_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, vp, i64p, i32p, vp, i64p,
                                           i32p, vp, i64p, i64p, vp, vp]),
        "mpzmm_server_create": (C.c_int, [C.POINTER(vp), C.c_int64, C.c_int, C.c_int]),
        "mpzmm_server_submit": (C.c_int, [vp, C.POINTER(Product), C.POINTER(C.c_uint64)]),
        "mpzmm_server_wait": (C.c_int, [vp, C.c_uint64, C.c_int64]),
        "mpzmm_server_poll": (C.c_int, [vp, C.c_uint64, C.POINTER(C.c_int)]),
        "mpzmm_server_ticket_times": (C.c_int, [vp, C.c_uint64, i64p, i64p, i64p]),
        "mpzmm_server_release": (C.c_int, [vp, C.c_uint64]),
        "mpzmm_server_stats": (C.c_int, [vp, i64p, i64p, i64p]),
        "mpzmm_server_set_admission_window": (C.c_int, [vp, C.c_int64]),
        "mpzmm_server_destroy": (None, [vp]),
        "mpzmm_server_phase_ns": (C.c_int, [vp, i64p]),
        "mpzmm_server_phase_max_ns": (C.c_int, [vp, i64p]),
        "mpzmm_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(vp)]),
        "mpzmm_host_free": (C.c_int, [vp]),
        "mpzmm_host_register": (C.c_int, [vp, C.c_size_t]),
        "mpzmm_host_unregister": (C.c_int, [vp]),
        "mpzmm_batch_stats": (C.c_int, [i64p, i64p, i64p]),
        "mpzmm_batch_timeline": (C.c_int, [C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int)]),
        "mpzmm_batch_chunks": (C.c_int, [C.c_int, i64p, C.c_int64, i64p, C.c_int,
                                         C.POINTER(C.c_int)]),
        "mpzmm_chain_output_limbs": (C.c_int64, [C.c_int, C.POINTER(Matrix)]),
        "mpzmm_chain": (C.c_int, [C.c_int, C.POINTER(Matrix), u64p, i64p, i64p, i32p, vp]),
        "mpzmm_mod_create": (C.c_int, [C.POINTER(vp), u64p, C.c_int32, C.c_int64]),
        "mpzmm_mod_limbs": (C.c_int64, [vp]),
        "mpzmm_mod_batch": (C.c_int, [vp, C.c_int, u64p, i64p, i32p, u64p, i64p, i64p, i32p, vp]),
        "mpzmm_mod_destroy": (None, [vp]),
        "mpzmm_mod_mpz": (C.c_int, [vp, vp, vp, C.c_int, vp]),
        "mpzmm_choose_params": (C.c_int, [C.c_int64, C.c_int64, C.c_int, C.POINTER(C.c_int),
                                          C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status: int) -> None:
    if status != MPZMM_OK:
        raise MpzmmError(status, lib().mpzmm_last_error().decode(errors="replace"))
