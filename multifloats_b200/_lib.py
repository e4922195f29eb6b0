"""ctypes binding of libmultifloats_cuda.so (the C ABI in include/multifloats_cuda.h).

The shared library is built in-tree (``python -m multifloats_b200.build``).  There
is no fallback: if the library is missing or fails to load, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmultifloats_cuda.so")


class float64x2(C.Structure):
    """The reference's interchange struct: limbs[0] = hi, limbs[1] = lo."""

    _fields_ = [("hi", C.c_double), ("lo", C.c_double)]


class complex64x2(C.Structure):
    _fields_ = [("re", float64x2), ("im", float64x2)]


class gemm_desc(C.Structure):
    """mfcuda_gemm_desc: device pointers and sizes of one batched product."""

    _fields_ = [("a", C.c_void_p), ("b", C.c_void_p), ("c", C.c_void_p),
                ("m", C.c_int64), ("k", C.c_int64), ("n", C.c_int64)]


class MFCudaError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        msg = _lib.mfcuda_error_string(code).decode() if _lib is not None else str(code)
        super().__init__(f"{where}: {msg} (code {code})")


P = C.c_void_p
I64 = C.c_int64

# name -> (restype, argtypes)
SIGNATURES = {
    "mfcuda_last_error": (C.c_int, []),
    "mfcuda_error_string": (C.c_char_p, [C.c_int]),
    "mfcuda_version": (C.c_char_p, []),
    # drop-in
    "matmuldd_mm": (None, [P, P, P, I64, I64, I64, I64]),
    "matmuldd_mv": (None, [P, P, P, I64, I64, I64]),
    "matmuldd_vm": (None, [P, P, P, I64, I64, I64]),
    "matmulf64x2_mm": (None, [P, P, P, I64, I64, I64, I64]),
    "matmulf64x2_mv": (None, [P, P, P, I64, I64, I64]),
    "matmulf64x2_vm": (None, [P, P, P, I64, I64, I64]),
    "cmatmuldd_mm": (None, [P, P, P, I64, I64, I64, I64]),
    "expdd_array": (None, [P, P, I64]),
    "logdd_array": (None, [P, P, I64]),
    "sindd_array": (None, [P, P, I64]),
    "cosdd_array": (None, [P, P, I64]),
    "sqrtdd_array": (None, [P, P, I64]),
    "sumdd_array": (float64x2, [P, I64]),
    "dotdd_array": (float64x2, [P, P, I64, I64]),
    "norm2dd_array": (float64x2, [P, I64]),
    "csumdd_array": (complex64x2, [P, I64]),
    "cdotdd_array": (complex64x2, [P, P, I64, I64]),
    "cnorm2dd_array": (float64x2, [P, I64]),
    "matmuldd_mm_split": (None, [P, P, P, I64, I64, I64, C.c_int, C.POINTER(C.c_double)]),
    "mfcuda_split_workspace_size": (C.c_size_t, [I64, I64, I64]),
    "mfcuda_crt_workspace_size": (C.c_size_t, [I64, I64, I64, C.c_int]),
    "mfcuda_matmuldd_mm_crt": (C.c_int, [P, P, P, I64, I64, I64, C.c_int, C.c_double, P, C.c_size_t, P, P]),
    "matmuldd_mm_crt": (None, [P, P, P, I64, I64, I64, C.c_int, C.POINTER(C.c_double)]),
    "mfcuda_crt_bound": (C.c_double, [C.c_int, C.c_int, C.c_int, I64]),
    "mfcuda_ccrt_workspace_size": (C.c_size_t, [I64, I64, I64, C.c_int]),
    "mfcuda_cmatmuldd_mm_crt": (C.c_int, [P, P, P, I64, I64, I64, C.c_int, C.c_double, P, C.c_size_t, P, P]),
    "cmatmuldd_mm_crt": (None, [P, P, P, I64, I64, I64, C.c_int, C.POINTER(C.c_double)]),
    "mfcuda_csplit_workspace_size": (C.c_size_t, [I64, I64, I64]),
    "mfcuda_cmatmuldd_mm_split": (C.c_int, [P, P, P, I64, I64, I64, C.c_int, C.c_double, P, C.c_size_t,
                                            P, P]),
    "cmatmuldd_mm_split": (None, [P, P, P, I64, I64, I64, C.c_int, C.POINTER(C.c_double)]),
    "mfcuda_batch_create_gemm": (C.c_int, [P, I64, C.c_int, I64, C.c_int, C.c_double, C.c_int, C.POINTER(P)]),
    "mfcuda_batch_create_cgemm": (C.c_int, [P, I64, C.c_int, I64, C.c_int, C.c_double, C.c_int, C.POINTER(P)]),
    "mfcuda_batch_create_unary": (C.c_int, [C.c_int, P, P, P, I64, C.POINTER(P)]),
    "mfcuda_batch_run": (C.c_int, [P, P]),
    "mfcuda_batch_status": (C.c_int, [P]),
    "mfcuda_batch_config": (I64, [P, I64]),
    "mfcuda_batch_work_items": (I64, [P]),
    "mfcuda_batch_kchunk": (I64, [P]),
    "mfcuda_batch_destroy": (None, [P]),
    "mfcuda_unary_dd_ragged": (C.c_int, [C.c_int, P, P, P, I64, P]),
    "mfcuda_phase_profile_begin": (None, []),
    "mfcuda_phase_profile_end": (C.c_int, [C.POINTER(C.c_double), C.POINTER(I64)]),
    "mfcuda_set_wait_limit_ns": (C.c_uint64, [C.c_uint64]),
    "mfcuda_shard_bounds": (None, [I64, C.c_int, C.c_int, C.POINTER(I64), C.POINTER(I64)]),
    "mfcuda_nccl_available": (C.c_int, []),
    "mfcuda_matmuldd_mm_nccl": (C.c_int, [C.c_int, P, P, P, I64, I64, I64, I64, C.c_double, C.c_int, P,
                                          C.c_size_t, P, P, P]),
    "mfcuda_reduce_nccl": (C.c_int, [C.c_int, P, P, I64, I64, P, P, P]),
    "mfcuda_timeout_status": (C.c_int, [C.c_int]),
    "mfcuda_matmuldd_mm_split": (C.c_int, [P, P, P, I64, I64, I64, C.c_int, C.c_double, P, C.c_size_t,
                                           P, P]),
    # device-pointer API
    "mfcuda_matmuldd_mm": (C.c_int, [P, P, P, I64, I64, I64, I64, P]),
    "mfcuda_matmuldd_mv": (C.c_int, [P, P, P, I64, I64, I64, P]),
    "mfcuda_matmuldd_vm": (C.c_int, [P, P, P, I64, I64, I64, P]),
    "mfcuda_cmatmuldd_mm": (C.c_int, [P, P, P, I64, I64, I64, I64, P]),
    "mfcuda_unary_dd": (C.c_int, [C.c_int, P, P, I64, P]),
    "mfcuda_sincos_dd": (C.c_int, [P, P, P, I64, P]),
    "mfcuda_cexpi_dd": (C.c_int, [P, P, I64, P]),
    "mfcuda_cexp_dd": (C.c_int, [P, P, I64, P]),
    "exp2dd_array": (None, [P, P, I64]),
    "log2dd_array": (None, [P, P, I64]),
    "log10dd_array": (None, [P, P, I64]),
    "sincosdd_array": (None, [P, P, P, I64]),
    "cexpidd_array": (None, [P, P, I64]),
    "cexpdd_array": (None, [P, P, I64]),
    "mfcuda_reduce_workspace_size": (C.c_size_t, [I64]),
    "mfcuda_reduce_geometry": (None, [I64, C.POINTER(I64), C.POINTER(I64)]),
    "mfcuda_sumdd": (C.c_int, [P, I64, P, P, C.c_size_t, P]),
    "mfcuda_dotdd": (C.c_int, [P, P, I64, I64, P, P, C.c_size_t, P]),
    "mfcuda_dotdd_noalloc": (C.c_int, [P, P, I64, I64, P, P]),
    "mfcuda_reduce_partial_values": (C.c_int, [C.c_int]),
    "mfcuda_reduce_partial": (C.c_int, [C.c_int, P, P, I64, I64, P, P, C.c_size_t, P]),
    "mfcuda_reduce_combine": (C.c_int, [C.c_int, P, I64, P, P]),
    "mfcuda_norm2dd": (C.c_int, [P, I64, P, P, C.c_size_t, P]),
    "mfcuda_csumdd": (C.c_int, [P, I64, P, P, C.c_size_t, P]),
    "mfcuda_cdotdd": (C.c_int, [P, P, I64, I64, P, P, C.c_size_t, P]),
    "mfcuda_cnorm2dd": (C.c_int, [P, I64, P, P, C.c_size_t, P]),
    # BLAS-style shims
    "mfcuda_wgemm_dd": (C.c_int, [C.c_char, C.c_char, I64, I64, I64, P, P, I64, P, I64, P, P, I64, P, P]),
    "mfcuda_wtrsm_dd": (C.c_int, [C.c_char, C.c_char, C.c_char, C.c_char, I64, I64, P, P, I64, P, I64,
                                  P, P]),
    "wgemm_": (None, [P, P, P, P, P, P, P, P, P, P, P, P, P, C.c_size_t, C.c_size_t]),
    "wtrsm_": (None, [P, P, P, P, P, P, P, P, P, P, P, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t]),
}

_lib = None
_lock = threading.Lock()


def lib():
    """Load (once) and return the CUDA library; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m multifloats_b200.build`")
            handle = C.CDLL(LIB_PATH, mode=C.RTLD_LOCAL)
            for name, (res, args) in SIGNATURES.items():
                if not hasattr(handle, name):
                    continue  # optional symbol; tests check the exported list
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
    return _lib


def check(code: int, where: str) -> None:
    if code != 0:
        raise MFCudaError(code, where)


def check_last(where: str) -> None:
    check(lib().mfcuda_last_error(), where)
