"""GPU tests of the failure paths, made to fail on the host side or by a
shortened wait limit -- no kernel is broken and nothing faults:

  * MFCUDA_FAIL_ALLOC=1 makes the first staging allocation of a process
    report MFCUDA_ERR_ALLOC without calling the allocator: the drop-in
    symbols (matmuldd_mm, expdd_array, matmuldd_mm_crt) latch it in
    mfcuda_last_error() and the next call in the same process succeeds with
    the reference's results;
  * mfcuda_set_wait_limit_ns(1) makes the bounded waits of the tensor-core
    kernels give up almost at once: the split and CRT calls (single-CTA
    kernel, m <= 128) and a batch plan report MFCUDA_ERR_TIMEOUT, the device
    record (mfcuda_timeout_status) shows it until cleared, and once the
    default limit is restored the same calls are bit-identical to the oracle
    again in the same context.  The operands are long enough in K that the
    first accumulator takes tens of microseconds: a wait always outlasts
    the shortened limit."""
import ctypes as C
import os
import subprocess
import sys

import pytest

from conftest import ROOT, to_dev, to_host
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ERR_ALLOC, ERR_TIMEOUT = 3, 5

_CHILD = r"""
import ctypes as C, sys
sys.path.insert(0, {root!r})
import numpy as np
from multifloats_b200 import _lib
from multifloats_b200 import workloads as W
from oracle import oracle as O
L = _lib.lib()
what = {what!r}
p = lambda a: a.ctypes.data
if what == "matmuldd_mm":
    m, k, n = 70, 90, 50
    a, b = W.dd_uniform(m * k, 1), W.dd_uniform(k * n, 2)
    want = O.matmul_mm(a, b, m, k, n, 8)
    call = lambda c: L.matmuldd_mm(p(a), p(b), p(c), m, k, n, 8)
    size = 2 * m * n
elif what == "expdd_array":
    x = W.dd_exp_inputs(5000, 3)
    want = O.unary("exp", x)
    call = lambda y: L.expdd_array(p(x), p(y), 5000)
    size = x.size
else:
    m, k, n = 200, 300, 150
    a = W.dd_rowcol_scaled(m, k, 16, "row", 4)
    b = W.dd_rowcol_scaled(k, n, 16, "col", 5)
    want, _ = O.crt_gemm(a, b, m, k, n)
    bound = C.c_double()
    call = lambda c: L.matmuldd_mm_crt(p(a), p(b), p(c), m, k, n, 0, C.byref(bound))
    size = 2 * m * n
out = np.full(size, 7.0)
call(out)
first = L.mfcuda_last_error()
out2 = np.full(size, 7.0)
call(out2)
second = L.mfcuda_last_error()
print(first, second, int(O.same_bits(out2, want).all()))
"""


@pytest.mark.parametrize("what", ["matmuldd_mm", "expdd_array", "matmuldd_mm_crt"])
def test_dropin_latches_alloc_failure_then_recovers(what):
    env = dict(os.environ, MFCUDA_FAIL_ALLOC="1")
    proc = subprocess.run([sys.executable, "-c", _CHILD.format(root=ROOT, what=what)], env=env,
                          capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stderr
    first, second, exact = (int(v) for v in proc.stdout.split()[-3:])
    assert first == ERR_ALLOC, first
    assert second == 0 and exact == 1


def _stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.fixture
def short_waits(cuda_lib):
    """A 1 ns wait limit for the test, the default restored afterwards."""
    cuda_lib.mfcuda_timeout_status(1)
    prev = cuda_lib.mfcuda_set_wait_limit_ns(1)
    try:
        yield
    finally:
        cuda_lib.mfcuda_set_wait_limit_ns(prev)
        import torch

        torch.cuda.synchronize()
        cuda_lib.mfcuda_timeout_status(1)


def _call(L, form, dA, dB, dC, m, k, n):
    info = (C.c_int * 4)()
    sym = L.mfcuda_matmuldd_mm_crt if form == "crt" else L.mfcuda_matmuldd_mm_split
    rc = sym(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), m, k, n, 0, 8.0, None, 0, info, _stream())
    return rc, list(info)


@pytest.mark.parametrize("form", ["split", "crt"])
def test_wait_limit_expires_then_default_is_exact(cuda_lib, dev, short_waits, form):
    import torch

    m, k, n = 96, 73 * 128, 256  # m <= 128: the single-CTA tensor-core kernel
    a = W.dd_rowcol_scaled(m, k, 8, "row", 31)
    b = W.dd_rowcol_scaled(k, n, 8, "col", 32)
    dA, dB = to_dev(a, dev), to_dev(b, dev)
    dC = torch.zeros(2 * m * n, dtype=torch.float64, device=dev)
    rc, _ = _call(cuda_lib, form, dA, dB, dC, m, k, n)
    assert rc == ERR_TIMEOUT, rc
    torch.cuda.synchronize()
    assert cuda_lib.mfcuda_timeout_status(0) == ERR_TIMEOUT
    assert cuda_lib.mfcuda_timeout_status(1) == ERR_TIMEOUT  # read and clear
    assert cuda_lib.mfcuda_timeout_status(0) == 0
    # the context is intact: with the default limit the same kernels are exact
    # (a shorter K keeps the oracle quick)
    assert cuda_lib.mfcuda_set_wait_limit_ns(0) == 1
    k = 600
    a, b = a.reshape(-1, m, 2)[:k].reshape(-1), b.reshape(n, -1, 2)[:, :k].reshape(-1)
    dA, dB = to_dev(a, dev), to_dev(b, dev)
    rc, info = _call(cuda_lib, form, dA, dB, dC, m, k, n)
    assert rc == 0
    if form == "crt":
        want, winfo = O.crt_gemm(a, b, m, k, n)
        assert info == winfo
    else:
        want, winfo = O.split_gemm(a, b, m, k, n)
        assert tuple(info[:3]) == winfo
    assert O.same_bits(to_host(dC), want).all()
    assert cuda_lib.mfcuda_timeout_status(0) == 0


def test_batch_plan_captures_the_wait_limit(cuda_lib, dev, short_waits):
    """A batch plan created under the short limit gives up its waits on every
    run (the limit is captured with the graph); a plan created after the
    default is restored is exact."""
    from test_gpu_batched import Batch

    bt = Batch(cuda_lib, dev, [(100, 73 * 128, 256), (64, 4000, 128)], 8100, W.dd_uniform)
    p = bt.plan(2)
    try:
        assert cuda_lib.mfcuda_batch_run(p, _stream()) == 0
        assert cuda_lib.mfcuda_batch_status(p) == ERR_TIMEOUT
    finally:
        cuda_lib.mfcuda_batch_destroy(p)
    assert cuda_lib.mfcuda_timeout_status(1) == ERR_TIMEOUT
    cuda_lib.mfcuda_set_wait_limit_ns(0)
    shapes = [(100, 700, 256), (64, 400, 128)]
    bt = Batch(cuda_lib, dev, shapes, 8200, W.dd_uniform)
    p = bt.plan(2)
    try:
        bt.run(p)
        for i, (m, k, n) in enumerate(shapes):
            want, _ = O.crt_gemm(bt.hA[i], bt.hB[i], m, k, n)
            assert O.same_bits(bt.result(i), want).all(), i
    finally:
        cuda_lib.mfcuda_batch_destroy(p)
    assert cuda_lib.mfcuda_timeout_status(0) == 0

