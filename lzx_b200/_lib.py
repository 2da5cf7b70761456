"""ctypes binding of the lattice_cuda C ABI (``include/lattice_cuda.h``).

The shared library is built in-tree (``lzx_b200/_build/liblattice_cuda.so``)
by :func:`lzx_b200.build.build`.  There is no CPU fallback: if the library is
missing or no sm_100 device is usable, calls raise :class:`LatticeCudaError`.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liblattice_cuda.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "lattice_cuda.h")

LC_OK = 0
LC_ERR_LENGTH_MISMATCH = 1
LC_ERR_ADICITY_TOO_SMALL = 2
LC_ERR_DIMENSION_MISMATCH = 3
LC_ERR_NORM_EXCEEDED = 4
LC_ERR_COMMITMENT_MISMATCH = 5
LC_ERR_NON_CANONICAL = 6
LC_ERR_INVALID_ARGUMENT = 7
LC_ERR_UNSUPPORTED = 8
LC_ERR_CUDA = 9
LC_ERR_OUT_OF_MEMORY = 10
LC_ERR_TIMEOUT = 11
LC_ERR_NO_DEVICE = 12
LC_ERR_LOG_N_OUT_OF_RANGE = 13
LC_ERR_GENERATOR_INVALID = 14

LC_KEY_TENSOR_I8 = 1
LC_ENGINE_NTT = 0
LC_ENGINE_TENSOR_I8 = 1
LC_PRODUCTS_INT64 = 0
LC_PRODUCTS_TENSOR = 1
LC_BATCH_GRAPH = 1


class LatticeCudaError(RuntimeError):
    """A non-zero lc_status returned by the C ABI."""

    def __init__(self, status: int, where: str = ""):
        self.status = status
        msg = _status_string(status)
        super().__init__(f"{where}: {msg} (status {status})" if where else msg)


_lock = threading.Lock()
_lib = None


def _status_string(status: int) -> str:
    try:
        return lib().lc_status_string(status).decode()
    except Exception:  # library itself unavailable
        return f"status {status}"


def _declare(L):
    P, sz, u32, i32 = C.c_void_p, C.c_size_t, C.c_uint32, C.c_int
    U32P = C.POINTER(C.c_uint32)
    sigs = {
        "lc_version": (C.c_char_p, []),
        "lc_status_string": (C.c_char_p, [i32]),
        "lc_device_available": (i32, []),
        "lc_ntt_plan_create_u32": (i32, [u32, U32P, U32P, U32P, u32, C.POINTER(P)]),
        "lc_ntt_plan_create_goldilocks": (i32, [u32, C.POINTER(P)]),
        "lc_ntt_plan_destroy": (None, [P]),
        "lc_ntt_plan_info": (i32, [P, U32P, U32P, U32P]),
        "lc_ntt_forward": (i32, [P, P, P, sz, P]),
        "lc_ntt_inverse": (i32, [P, P, P, sz, P]),
        "lc_ntt_forward_host": (i32, [P, P, P, sz]),
        "lc_ntt_inverse_host": (i32, [P, P, P, sz]),
        "lc_ntt_plan_check": (i32, [P, P]),
        "lc_ntt_plan_set_variant": (i32, [P, i32]),
        "lc_ajtai_key_create": (i32, [P, u32, u32, P, i32, C.POINTER(P)]),
        "lc_ajtai_key_destroy": (None, [P]),
        "lc_ajtai_key_info": (i32, [P, U32P, U32P, U32P]),
        "lc_ajtai_commit": (i32, [P, P, sz, P, P]),
        "lc_ajtai_commit_i8": (i32, [P, P, sz, P, P]),
        "lc_ajtai_commit_host": (i32, [P, P, sz, P]),
        "lc_ajtai_commit_i8_host": (i32, [P, P, sz, P]),
        "lc_ajtai_key_check": (i32, [P, P]),
        "lc_ajtai_commit_noalloc": (i32, [P, P, sz, P, P]),
        "lc_ajtai_key_create_ex": (i32, [P, u32, u32, P, i32, u32, C.POINTER(P)]),
        "lc_ajtai_key_set_engine": (i32, [P, i32]),
        "lc_ajtai_key_get_engine": (i32, [P]),
        "lc_ajtai_key_set_fused": (i32, [P, i32]),
        "lc_tc_i8_rate": (i32, [u32, i32, C.POINTER(C.c_double), C.POINTER(C.c_float)]),
        "lc_ajtai_key_get_fused": (i32, [P]),
        "lc_ajtai_key_set_slot_products": (i32, [P, i32]),
        "lc_ajtai_key_get_slot_products": (i32, [P]),
        "lc_ajtai_commit_u8": (i32, [P, P, sz, P, P]),
        "lc_ajtai_commit_u8_host": (i32, [P, P, sz, P]),
        "lc_decomp_b": (i32, [P, sz, u32, P, P]),
        "lc_gadget_decompose": (i32, [P, sz, u32, u32, P, P, P]),
        "lc_crt_residues": (i32, [P, P, sz, P, P]),
        "lc_fold_pipeline_create": (i32, [P, P, i32, C.POINTER(P)]),
        "lc_fold_pipeline_buffers": (i32, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
        "lc_fold_pipeline_run": (i32, [P, P]),
        "lc_fold_pipeline_check": (i32, [P, P]),
        "lc_fold_pipeline_destroy": (None, [P]),
        "lc_ajtai_key_view": (i32, [P, u32, u32, C.POINTER(P)]),
        "lc_uniform_from_seed": (i32, [P, P, sz, P, sz, C.c_uint64, sz, P, P]),
        "lc_ntt_forward_partial": (i32, [P, P, P, sz, u32, P]),
        "lc_pack_field_elements": (i32, [P, sz, u32, sz, P, P]),
        "lc_ntt_complete_partial": (i32, [P, P, P, sz, u32, P]),
        "lc_ajtai_key_from_seed": (i32, [P, u32, u32, P, C.POINTER(P)]),
        "lc_batch_create": (i32, [P, u32, P, u32, u32, C.POINTER(P)]),
        "lc_batch_set_config": (i32, [P, u32, u32, u32]),
        "lc_batch_get_config": (i32, [P, U32P, U32P, U32P]),
        "lc_batch_set_products": (i32, [P, i32]),
        "lc_batch_get_products": (i32, [P]),
        "lc_batch_info": (i32, [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), U32P]),
        "lc_batch_run": (i32, [P, P]),
        "lc_batch_check": (i32, [P, P]),
        "lc_batch_destroy": (None, [P]),
        "lc_synth_fill": (i32, [i32, C.c_uint64, C.c_uint64, u32, P, sz, sz, P]),
        "lc_quad50_plan_create": (i32, [C.c_uint64, u32, C.c_uint64, u32, C.POINTER(P)]),
        "lc_quad50_plan_destroy": (None, [P]),
        "lc_quad50_plan_info": (i32, [P, P, P]),
        "lc_quad50_forward": (i32, [P, P, P, sz, P]),
        "lc_quad50_inverse": (i32, [P, P, P, sz, P]),
        "lc_quad50_slotwise_mul": (i32, [P, P, P, P, sz, P]),
        "lc_quad50_mul": (i32, [P, P, P, P, sz, P]),
        "lc_quad50_mul_host": (i32, [P, P, P, P, sz]),
        "lc_lb_key_random": (i32, [sz, C.c_uint64, P, u32, C.POINTER(P)]),
        "lc_lb_key_create": (i32, [sz, P, u32, P, C.POINTER(P)]),
        "lc_lb_key_destroy": (None, [P]),
        "lc_lb_key_info": (i32, [P, P, P, P, P]),
        "lc_lb_ntt": (i32, [P, u32, P, P, sz, P]),
        "lc_lb_commit": (i32, [P, P, u32, P, P, P, P]),
        "lc_lb_commit_host": (i32, [P, P, u32, P, P, P]),
        "lc_lb_random_elems": (i32, [sz, C.c_uint64, P]),
    }
    optional = {
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    for name, (res, args) in optional.items():
        if hasattr(L, name):
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
    return L


def lib():
    """Load (once) the in-tree CUDA library; raise if it is not built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise LatticeCudaError(
                    LC_ERR_NO_DEVICE,
                    f"lattice_cuda library not built ({LIB_PATH}); run lzx_b200.build.build()")
            _lib = _declare(C.CDLL(LIB_PATH))
        return _lib


def check(status: int, where: str = "") -> None:
    if status != LC_OK:
        raise LatticeCudaError(status, where)


def declared_functions() -> list[str]:
    """Names of every entry point declared with LC_API in include/*.h."""
    import glob
    import re
    names = []
    for h in sorted(glob.glob(os.path.join(os.path.dirname(HEADER), "*.h"))):
        src = open(h).read()
        names += re.findall(r"LC_API\s+[\w\s\*]+?\b(lc_\w+)\s*\(", src)
    return names
