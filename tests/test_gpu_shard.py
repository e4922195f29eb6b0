"""The NCCL-sharded C entry points on one GPU (a one-rank communicator: the
only GPU count a test here can have).  Column panels of one product and
sharded reductions go through mfcuda_matmuldd_mm_nccl / mfcuda_reduce_nccl
and must equal the single-device calls bit for bit (the multi-rank panel
arithmetic and the rank-order fold are covered on the CPU by
tests/test_dist.py and tests/test_shard_bounds.py)."""
import ctypes as C

import numpy as np
import pytest

from conftest import to_dev, to_host
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PLAIN, SPLIT, CRT = 0, 1, 2
PANELS, GATHER = 1, 2


@pytest.fixture(scope="module")
def comm(cuda_lib, dev):
    from multifloats_b200.nccl_comm import NcclComm

    assert cuda_lib.mfcuda_nccl_available() == 1
    c = NcclComm.single(0)
    yield c
    c.close()


def _stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("form,flags", [(PLAIN, 0), (SPLIT, GATHER), (CRT, 0), (CRT, PANELS), (CRT, GATHER)])
def test_product_equals_single_call(cuda_lib, dev, comm, form, flags):
    import torch

    m, k, n = 300, 260, 520
    a = W.dd_rowcol_scaled(m, k, 16, "row", 5)
    b = W.dd_rowcol_scaled(k, n, 16, "col", 6)
    dA, dB = to_dev(a, dev), to_dev(b, dev)
    dC = torch.full((2 * m * n,), float("nan"), dtype=torch.float64, device=dev)
    info = (C.c_int * 4)()
    param = 8 if form == PLAIN else 0
    rc = cuda_lib.mfcuda_matmuldd_mm_nccl(form, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), m, k, n, param, 8.0,
                                          flags, None, 0, info, comm.handle, _stream())
    assert rc == 0, cuda_lib.mfcuda_error_string(rc)
    got = to_host(dC)
    if form == PLAIN:
        want = O.matmul_mm(a, b, m, k, n, 8)
    elif form == SPLIT:
        want, winfo = O.split_gemm(a, b, m, k, n)
        assert tuple(info[:3]) == winfo
    else:
        want, winfo = O.crt_gemm(a, b, m, k, n)
        assert list(info) == winfo
    assert O.same_bits(got, want).all()


def test_k_zero_and_bad_arguments(cuda_lib, dev, comm):
    import torch

    c = torch.full((2 * 6,), 5.0, dtype=torch.float64, device=dev)
    a = torch.zeros(2, dtype=torch.float64, device=dev)
    assert cuda_lib.mfcuda_matmuldd_mm_nccl(CRT, a.data_ptr(), a.data_ptr(), c.data_ptr(), 2, 0, 3, 0, 8.0, 0,
                                            None, 0, None, comm.handle, _stream()) == 0
    assert (to_host(c) == 0).all()
    assert cuda_lib.mfcuda_matmuldd_mm_nccl(7, a.data_ptr(), a.data_ptr(), c.data_ptr(), 2, 0, 3, 0, 8.0, 0, None,
                                            0, None, comm.handle, _stream()) == 1
    assert cuda_lib.mfcuda_matmuldd_mm_nccl(CRT, a.data_ptr(), a.data_ptr(), c.data_ptr(), 2, 0, 3, 0, 8.0,
                                            PANELS | GATHER, None, 0, None, comm.handle, _stream()) == 1
    assert cuda_lib.mfcuda_matmuldd_mm_nccl(CRT, a.data_ptr(), a.data_ptr(), c.data_ptr(), 2, 0, 3, 0, 8.0, 0,
                                            None, 0, None, None, _stream()) == 1


@pytest.mark.parametrize("kind,code", [("sum", 0), ("dot", 1), ("norm2", 2), ("csum", 3), ("cdot", 4),
                                       ("cnorm2", 5)])
def test_reduction_equals_rank_order_fold(cuda_lib, dev, comm, kind, code):
    import torch

    n = 100003
    per = 2 if kind.startswith("c") else 1
    x = W.dd_uniform(per * n, seed=31)
    y = W.dd_uniform(per * n, seed=32)
    out = torch.empty(4, dtype=torch.float64, device=dev)
    dx, dy = to_dev(x, dev), to_dev(y, dev)  # held: the call runs asynchronously on the stream
    rc = cuda_lib.mfcuda_reduce_nccl(code, dx.data_ptr(), dy.data_ptr(), n, 8, out.data_ptr(), comm.handle,
                                     _stream())
    assert rc == 0
    nd = 4 if kind in ("csum", "cdot") else 2
    want = O.reduce_combine(kind, O.reduce_partial(kind, x, y if "dot" in kind else None, 8))
    assert O.same_bits(to_host(out)[:nd], want).all()
