"""mfcuda_dotdd_noalloc: the dot product for callers that cannot let a library
allocate device memory (an application that owns the whole GPU memory through
its own pool, or a latency-critical path where cudaMalloc / cudaFree would
synchronise the device).  Its block partials live in a fixed array inside the
library, so it must give exactly what mfcuda_dotdd gives -- bit for bit, the
tolerance the reduction tests use -- call after call, reject sizes its array
cannot hold, and never reach the library's allocator.

This file is named so that pytest collects it last."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, to_dev, to_host
from multifloats_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAX_N = 1024 * 4096  # capacity of the fixed partials array


def _dot_existing(L, a, b, n, ri, stream):
    import torch

    out = torch.empty(2, dtype=torch.float64, device=a.device)
    rc = L.mfcuda_dotdd(a.data_ptr(), b.data_ptr(), n, ri, out.data_ptr(), None, 0, stream)
    assert rc == 0
    return to_host(out)


def _dot_noalloc(L, a, b, n, ri, stream):
    import torch

    out = torch.empty(2, dtype=torch.float64, device=a.device)
    rc = L.mfcuda_dotdd_noalloc(a.data_ptr(), b.data_ptr(), n, ri, out.data_ptr(), stream)
    assert rc == 0, rc
    return to_host(out)


def test_matches_existing_entry_point_on_consecutive_calls(cuda_lib, dev):
    import torch

    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # two calls in a row, the second smaller than the first so that stale
    # partials from the first call are still sitting in the shared array
    for n, ri, seed in [(MAX_N - 5, 8, 1), (123457, 3, 2)]:
        ha, hb = W.dd_uniform(n, seed=seed), W.dd_uniform(n, seed=seed + 100)
        a, b = to_dev(ha, dev), to_dev(hb, dev)
        got = _dot_noalloc(cuda_lib, a, b, n, ri, stream)
        want = _dot_existing(cuda_lib, a, b, n, ri, stream)
        assert O.same_bits(got, want).all(), (n, got, want)
        # and directly against the CPU restatement of the device's blocked order
        assert O.same_bits(got, O.reduce_blocked("dot", ha, hb, ri)).all(), n


def test_small_and_empty(cuda_lib, dev):
    import torch

    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for n in (0, 1, 4097):
        a = to_dev(W.dd_uniform(max(n, 1), seed=7), dev)
        b = to_dev(W.dd_uniform(max(n, 1), seed=8), dev)
        assert O.same_bits(_dot_noalloc(cuda_lib, a, b, n, 8, stream),
                           _dot_existing(cuda_lib, a, b, n, 8, stream)).all()


def test_capacity_edge(cuda_lib, dev):
    """n = 4,194,304 (one partial per slot of the array) is accepted and
    exact; one element more is rejected before anything is read or launched."""
    import torch

    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    ha, hb = W.dd_uniform(MAX_N, seed=21), W.dd_uniform(MAX_N, seed=22)
    a, b = to_dev(ha, dev), to_dev(hb, dev)
    got = _dot_noalloc(cuda_lib, a, b, MAX_N, 8, stream)
    assert O.same_bits(got, O.reduce_blocked("dot", ha, hb, 8)).all()
    out = torch.full((2,), 7.0, dtype=torch.float64, device=dev)
    for n in (MAX_N + 1, MAX_N + 4096):
        rc = cuda_lib.mfcuda_dotdd_noalloc(a.data_ptr(), b.data_ptr(), n, 8, out.data_ptr(), None)
        assert rc == 7  # MFCUDA_ERR_UNSUPPORTED
    assert cuda_lib.mfcuda_error_string(7) == b"unsupported shape or parameter"
    assert (to_host(out) == 7.0).all()  # the rejected calls wrote nothing


_CHILD = r"""
import ctypes as C, sys
sys.path.insert(0, {root!r})
import numpy as np, torch
from multifloats_b200 import _lib
from multifloats_b200 import workloads as W
L = _lib.lib()
d = torch.device('cuda:0')
n = 50000
a = torch.from_numpy(W.dd_uniform(n, seed=3)).to(d)
b = torch.from_numpy(W.dd_uniform(n, seed=4)).to(d)
out = torch.empty(2, dtype=torch.float64, device=d)
rc1 = L.mfcuda_dotdd_noalloc(a.data_ptr(), b.data_ptr(), n, 8, out.data_ptr(), None)
rc2 = L.mfcuda_dotdd(a.data_ptr(), b.data_ptr(), n, 8, out.data_ptr(), None, 0, None)
torch.cuda.synchronize()
print(rc1, rc2)
"""


def test_never_reaches_the_allocator():
    # MFCUDA_FAIL_ALLOC=1 makes the library's first allocation attempt fail:
    # the no-allocation entry point still succeeds, the workspace-allocating
    # one reports MFCUDA_ERR_ALLOC.
    env = dict(os.environ, MFCUDA_FAIL_ALLOC="1")
    proc = subprocess.run([sys.executable, "-c", _CHILD.format(root=ROOT)], env=env,
                          capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stderr
    rc1, rc2 = (int(v) for v in proc.stdout.split()[-2:])
    assert rc1 == 0 and rc2 == 3
