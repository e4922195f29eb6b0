"""multifloats_b200: B200 (sm_100a) implementation of the multifloats double-double
array hot path -- compensated float64x2/complex64x2 matmul (plain FP64 and
split-INT8 on tcgen05 tensor cores), sum / dot_product / norm2 reductions and
elementwise exp / log / sin / cos / sqrt -- behind the C ABI declared in
include/multifloats_cuda.h.  This package is a thin ctypes mirror of that ABI.
"""
from .api import *  # noqa: F401,F403
from ._lib import LIB_PATH, MFCudaError, lib  # noqa: F401

__version__ = "0.1.0"
